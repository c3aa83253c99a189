// particles.cu -- particle kernels of the em2d step for sm_100a.
//
// Compiled with -fmad=false: no implicit FMA contraction.  The reference
// build (g++ -std=c++17) contracts nothing either and uses explicit fused
// multiply-adds only through ops::fma (utils.h:105-136), mirrored here with
// __fmaf_rn; division and square root stay IEEE (no fast-math).  A particle's
// push and move are therefore bit-identical to the reference.
#include "zpic_dev.cuh"

#include <algorithm>
#include <type_traits>

namespace zb {

// ---------------------------------------------------------------------------
// Per-particle physics
// ---------------------------------------------------------------------------

// 1 / Lorentz gamma (species.cpp:22-26).  1 / s rounded once is the
// correctly rounded reciprocal of s, so the reciprocal instruction gives the
// reference's quotient bit for bit.
__device__ __forceinline__ float rgamma( float ux, float uy, float uz ) {
    return __frcp_rn( sqrtf( __fmaf_rn( uz, uz, __fmaf_rn( uy, uy, __fmaf_rn( ux, ux, 1.0f ) ) ) ) );
}

// Linear interpolation of the staggered Yee fields (species.cpp:43-92).
// E, B point at cell (0,0) of float3 AoS tiles in shared memory.
__device__ __forceinline__ void interpolate_fld( const float * __restrict__ E, const float * __restrict__ B,
                                                 int ys, int i, int j, float xx, float xy,
                                                 float & ex, float & ey, float & ez,
                                                 float & bx, float & by, float & bz ) {
    const float s0x = 0.5f - xx, s1x = 0.5f + xx;
    const float s0y = 0.5f - xy, s1y = 0.5f + xy;
    const int hx = xx < 0, hy = xy < 0;
    const int ih = i - hx, jh = j - hy;
    const float s0xh = ( 1 - hx ) - xx, s1xh = ( hx ) + xx;
    const float s0yh = ( 1 - hy ) - xy, s1yh = ( hy ) + xy;
#define F3( A, c, k ) ( A[ 3 * ( c ) + ( k ) ] )
    ex = ( F3( E, ih +     j*ys, 0 ) * s0xh + F3( E, ih+1 +     j*ys, 0 ) * s1xh ) * s0y +
         ( F3( E, ih + (j+1)*ys, 0 ) * s0xh + F3( E, ih+1 + (j+1)*ys, 0 ) * s1xh ) * s1y;
    ey = ( F3( E, i  +    jh*ys, 1 ) * s0x  + F3( E, i+1  +    jh*ys, 1 ) * s1x  ) * s0yh +
         ( F3( E, i  + (jh+1)*ys, 1 ) * s0x + F3( E, i+1  + (jh+1)*ys, 1 ) * s1x  ) * s1yh;
    ez = ( F3( E, i  +     j*ys, 2 ) * s0x  + F3( E, i+1  +     j*ys, 2 ) * s1x  ) * s0y +
         ( F3( E, i  + (j+1)*ys, 2 ) * s0x  + F3( E, i+1  + (j+1)*ys, 2 ) * s1x  ) * s1y;
    bx = ( F3( B, i  +    jh*ys, 0 ) * s0x  + F3( B, i+1  +    jh*ys, 0 ) * s1x  ) * s0yh +
         ( F3( B, i  + (jh+1)*ys, 0 ) * s0x + F3( B, i+1  + (jh+1)*ys, 0 ) * s1x  ) * s1yh;
    by = ( F3( B, ih +     j*ys, 1 ) * s0xh + F3( B, ih+1 +     j*ys, 1 ) * s1xh ) * s0y +
         ( F3( B, ih + (j+1)*ys, 1 ) * s0xh + F3( B, ih+1 + (j+1)*ys, 1 ) * s1xh ) * s1y;
    bz = ( F3( B, ih +    jh*ys, 2 ) * s0xh + F3( B, ih+1 +    jh*ys, 2 ) * s1xh ) * s0yh +
         ( F3( B, ih + (jh+1)*ys, 2 ) * s0xh + F3( B, ih+1 + (jh+1)*ys, 2 ) * s1xh ) * s1yh;
#undef F3
}

// Relativistic Boris push with tangent-linearised rotation (species.cpp:117-178)
__device__ __forceinline__ void dudt_boris( float alpha, float ex, float ey, float ez,
                                            float bx, float by, float bz,
                                            float & ux, float & uy, float & uz, double & energy ) {
    ex *= alpha; ey *= alpha; ez *= alpha;
    float utx = ux + ex, uty = uy + ey, utz = uz + ez;
    {
        const float utsq = __fmaf_rn( utz, utz, __fmaf_rn( uty, uty, utx * utx ) );
        const float gamma = sqrtf( 1.0f + utsq );
        energy += (double) ( utsq / ( gamma + 1.0f ) );
        const float alpha_gamma = alpha / gamma;
        bx *= alpha_gamma; by *= alpha_gamma; bz *= alpha_gamma;
    }
    float vx = __fmaf_rn( bz, uty, utx );
    float vy = __fmaf_rn( bx, utz, uty );
    float vz = __fmaf_rn( by, utx, utz );
    vx = __fmaf_rn( -by, utz, vx );
    vy = __fmaf_rn( -bz, utx, vy );
    vz = __fmaf_rn( -bx, uty, vz );
    {
        // 2 / d (d >= 1): doubling is exact, so 2 * RN(1/d) = RN(2/d) bit for bit
        const float otsq = 2.0f * __frcp_rn( __fmaf_rn( bz, bz, __fmaf_rn( by, by, __fmaf_rn( bx, bx, 1.0f ) ) ) );
        bx *= otsq; by *= otsq; bz *= otsq;
    }
    utx = __fmaf_rn( bz, vy, utx );
    uty = __fmaf_rn( bx, vz, uty );
    utz = __fmaf_rn( by, vx, utz );
    utx = __fmaf_rn( -by, vz, utx );
    uty = __fmaf_rn( -bz, vx, uty );
    utz = __fmaf_rn( -bx, vy, utz );
    ux = utx + ex; uy = uty + ey; uz = utz + ez;
}

// Boris push with exact Euler-Rodrigues rotation (species.cpp:193-254)
__device__ __forceinline__ void dudt_boris_euler( float alpha, float ex, float ey, float ez,
                                                  float bx, float by, float bz,
                                                  float & ux, float & uy, float & uz, double & energy ) {
    ex *= alpha; ey *= alpha; ez *= alpha;
    const float utx = ux + ex, uty = uy + ey, utz = uz + ez;
    {
        const float utsq = __fmaf_rn( utz, utz, __fmaf_rn( uty, uty, utx * utx ) );
        const float gamma = sqrtf( 1.0f + utsq );
        energy += (double) ( utsq / ( gamma + 1.0f ) );
        const float alpha2_gamma = ( alpha * 2 ) / gamma;
        bx *= alpha2_gamma; by *= alpha2_gamma; bz *= alpha2_gamma;
    }
    const float bnorm = sqrtf( __fmaf_rn( bx, bx, __fmaf_rn( by, by, bz * bz ) ) );
    const float s = -( ( bnorm > 0 ) ? sinf( bnorm / 2 ) / bnorm : 1 );
    const float ra = cosf( bnorm / 2 );
    const float rb = bx * s, rc = by * s, rd = bz * s;
    const float r11 =     __fmaf_rn( ra, ra, rb * rb ) - __fmaf_rn( rc, rc, rd * rd );
    const float r12 = 2 * __fmaf_rn( rb, rc, ra * rd );
    const float r13 = 2 * __fmaf_rn( rb, rd, -ra * rc );
    const float r21 = 2 * __fmaf_rn( rb, rc, -ra * rd );
    const float r22 =     __fmaf_rn( ra, ra, rc * rc ) - __fmaf_rn( rb, rb, rd * rd );
    const float r23 = 2 * __fmaf_rn( rc, rd, ra * rb );
    const float r31 = 2 * __fmaf_rn( rb, rd, ra * rc );
    const float r32 = 2 * __fmaf_rn( rc, rd, -ra * rb );
    const float r33 =     __fmaf_rn( ra, ra, rd * rd ) - __fmaf_rn( rb, rb, -rc * rc );
    ux = __fmaf_rn( r11, utx, __fmaf_rn( r21, uty, r31 * utz ) ) + ex;
    uy = __fmaf_rn( r12, utx, __fmaf_rn( r22, uty, r32 * utz ) ) + ey;
    uz = __fmaf_rn( r13, utx, __fmaf_rn( r23, uty, r33 * utz ) ) + ez;
}

// Accumulation of one current contribution into the shared-memory tile
// current: FP32 or FP64 atomics, or fixed point.  Fixed point: the
// contribution arrives already multiplied by js (a power of two that keeps
// every contribution below 2^31 in magnitude, folded into the charge factors)
// and is rounded to an integer x; floor(x / 2^16) is added to a hi word and x
// itself (mod 2^32) to a second word jlo entries later, both with native
// shared-memory integer atomics.  Integer sums do not depend on the order of
// the additions; the hi sum cannot overflow and the low parts are recovered
// exactly for up to 2^16 additions per entry, and the kernel flushes the
// accumulators before that many.
struct JAcc { float js; int jlo; };
__device__ __forceinline__ void jadd( float * p, float v, JAcc ) { atomicAdd( p, v ); }
__device__ __forceinline__ void jadd( double * p, float v, JAcc ) { atomicAdd( p, (double) v ); }
__device__ __forceinline__ void jadd( int * p, float v, JAcc a ) {
    const int x = __float2int_rn( v );
    atomicAdd( p, x >> 16 );
    atomicAdd( reinterpret_cast<unsigned int *>( p + a.jlo ), (unsigned int) x );
}
// value of a fixed-point accumulator pair: hi = sum of floor(x / 2^16),
// full = sum of x mod 2^32, so full - hi * 2^16 (mod 2^32) is the sum of the
// low 16-bit parts, exact below 2^32 (up to 65537 additions).
__device__ __forceinline__ double jfix_value( int hi, unsigned int full, double inv ) {
    const unsigned int lo = full - ( (unsigned int) hi << 16 );
    return ( (double) hi * 65536.0 + (double) lo ) * inv;
}

// Charge-conserving current of one segment inside one cell (species.cpp:267-310),
// accumulated into the shared-memory tile current with shared atomics.
// hqx, hqy are half the reference's qnx, qny and qvz its q vz / 2, all times
// the fixed-point scale for the fixed-point tile current: powers of two, so
// every in-plane contribution is bit-identical to the reference's.  The
// out-of-plane weights are regrouped as a (c + d/2) + b (d - c/2) for the
// fixed-point current (a few roundings apart); FP32 and FP64 tile currents
// keep the reference's expression.
template < typename JT >
__device__ __forceinline__ void dep_current_seg( int ix, int iy, float x0x, float x0y, float x1x, float x1y,
                                                 float hqx, float hqy, float qvz, JT * J, int stride, JAcc ja ) {
    const float S0x0 = 0.5f - x0x, S0x1 = 0.5f + x0x;
    const float S1x0 = 0.5f - x1x, S1x1 = 0.5f + x1x;
    const float S0y0 = 0.5f - x0y, S0y1 = 0.5f + x0y;
    const float S1y0 = 0.5f - x1y, S1y1 = 0.5f + x1y;
    const float wl1 = hqx * ( x1x - x0x );
    const float wl2 = hqy * ( x1y - x0y );
    JT * Js = J + 3 * ( ix + stride * iy );
    const int s3 = 3 * stride;
    jadd( Js + 0,      wl1 * ( S0y0 + S1y0 ), ja );
    jadd( Js + 1,      wl2 * ( S0x0 + S1x0 ), ja );
    jadd( Js + 3 + 1,  wl2 * ( S0x1 + S1x1 ), ja );
    jadd( Js + s3 + 0, wl1 * ( S0y1 + S1y1 ), ja );
    if constexpr ( std::is_same<JT, int>::value ) {
        const float qp0 = qvz * __fmaf_rn( S1y0, 0.5f, S0y0 ), qq0 = qvz * __fmaf_rn( S0y0, -0.5f, S1y0 );
        const float qp1 = qvz * __fmaf_rn( S1y1, 0.5f, S0y1 ), qq1 = qvz * __fmaf_rn( S0y1, -0.5f, S1y1 );
        jadd( Js + 2,      __fmaf_rn( S0x0, qp0, S1x0 * qq0 ), ja );
        jadd( Js + 3 + 2,  __fmaf_rn( S0x1, qp0, S1x1 * qq0 ), ja );
        jadd( Js + s3 + 2, __fmaf_rn( S0x0, qp1, S1x0 * qq1 ), ja );
        jadd( Js + s3 + 5, __fmaf_rn( S0x1, qp1, S1x1 * qq1 ), ja );
    } else {
        jadd( Js + 2,      qvz * ( S0x0 * S0y0 + S1x0 * S1y0 + ( S0x0 * S1y0 - S1x0 * S0y0 ) / 2.0f ), ja );
        jadd( Js + 3 + 2,  qvz * ( S0x1 * S0y0 + S1x1 * S1y0 + ( S0x1 * S1y0 - S1x1 * S0y0 ) / 2.0f ), ja );
        jadd( Js + s3 + 2, qvz * ( S0x0 * S0y1 + S1x0 * S1y1 + ( S0x0 * S1y1 - S1x0 * S0y1 ) / 2.0f ), ja );
        jadd( Js + s3 + 5, qvz * ( S0x1 * S0y1 + S1x1 * S1y1 + ( S0x1 * S1y1 - S1x1 * S0y1 ) / 2.0f ), ja );
    }
}

// Split the trajectory of a particle that crosses at least one cell edge into
// two or three single-cell segments and deposit them (species.cpp:336-430
// split2d, crossing cases).  x1 = x0 + (dx, dy) before the cell correction.
// The split fractions use the approximate division __fdividef (2 ulp): they
// only place the split point on the cell edge, and the particle's own move
// stays exact.
template < typename JT >
__device__ __forceinline__ void deposit_crossing( int ix, int iy, float x0x, float x0y, float x1x, float x1y,
                                                  float dx, float dy, float qvz, float qnxx, float qnxy,
                                                  JT * J, int stride, JAcc ja ) {
    const int dix = ( ( x1x >= 0.5f ) - ( x1x < -0.5f ) );
    const int diy = ( ( x1y >= 0.5f ) - ( x1y < -0.5f ) );
    const int crossx = dix != 0, crossy = diy != 0;
    // first split: on x when x is crossed, else on y (selects, no branch)
    const float a0 = crossx ? x0x : x0y, b0 = crossx ? x0y : x0x;
    const float da = crossx ? dx : dy, db = crossx ? dy : dx;
    const float aint = crossx ? 0.5f * dix : 0.5f * diy;
    float eps = __fdividef( aint - a0, da );
    const float bint = b0 + db * eps;
    const float xint = crossx ? aint : bint, yint = crossx ? bint : aint;
    int v0x = ix, v0y = iy;  float v0x0 = x0x, v0y0 = x0y, v0x1 = xint, v0y1 = yint, v0q = qvz * eps;
    int v1x = ix + ( crossx ? dix : 0 ), v1y = iy + ( crossx ? 0 : diy );
    float v1x0 = crossx ? -xint : xint, v1y0 = crossx ? yint : -yint;
    float v1x1 = crossx ? x1x - dix : x1x, v1y1 = crossx ? x1y : x1y - diy;
    float v1q = qvz * ( 1 - eps );
    int v2x = 0, v2y = 0;    float v2x0 = 0, v2y0 = 0, v2x1 = 0, v2y1 = 0, v2q = 0;
    if ( crossx && crossy ) {
        const float yint2 = 0.5f * diy;
        if ( yint >= -0.5f && yint < 0.5f ) {
            eps = __fdividef( yint2 - yint, x1y - yint );
            const float xint2 = -xint + ( x1x - xint ) * eps;
            v2x = v1x; v2y = v1y + diy;
            v2x0 = xint2; v2y0 = -yint2;
            v2x1 = v1x1; v2y1 = v1y1 - diy;
            v2q = v1q * ( 1 - eps );
            v1x1 = xint2; v1y1 = yint2;
            v1q *= eps;
        } else {
            eps = __fdividef( yint2 - x0y, yint - x0y );
            const float xint2 = x0x + ( xint - x0x ) * eps;
            v2x = v0x; v2y = v0y + diy;
            v2x0 = xint2; v2y0 = -yint2;
            v2x1 = v0x1; v2y1 = v0y1 - diy;
            v2q = v0q * ( 1 - eps );
            v0x1 = xint2; v0y1 = yint2;
            v0q *= eps;
            v1y += diy;
            v1y0 -= diy;
            v1y1 -= diy;
        }
    }
    dep_current_seg( v0x, v0y, v0x0, v0y0, v0x1, v0y1, qnxx, qnxy, v0q, J, stride, ja );
    dep_current_seg( v1x, v1y, v1x0, v1y0, v1x1, v1y1, qnxx, qnxy, v1q, J, stride, ja );
    if ( crossx && crossy ) dep_current_seg( v2x, v2y, v2x0, v2y0, v2x1, v2y1, qnxx, qnxy, v2q, J, stride, ja );
}

// Per-warp ring of cell-crossing particles waiting for their split deposit.
constexpr int XQ = 64;                      // entries per warp (power of two)
struct CrossQueue {
    uint32_t cell[XQ];
    float x0x[XQ], x0y[XQ], dx[XQ], dy[XQ], qvz[XQ];
};

// Not inlined: the split deposit of a queued crossing is called from two
// places in the particle kernel, and one out-of-line copy keeps the kernel's
// instruction footprint (and instruction-cache misses) smaller -- 3 % faster.
template < typename JT >
__device__ __noinline__ void drain_entry( const CrossQueue & Q, int e, float qnxx, float qnxy, JT * J, int stride,
                                             JAcc ja ) {
    const uint32_t c = Q.cell[e];
    const float x0x = Q.x0x[e], x0y = Q.x0y[e], dx = Q.dx[e], dy = Q.dy[e];
    deposit_crossing( cell_x( c ), cell_y( c ), x0x, x0y, x0x + dx, x0y + dy, dx, dy, Q.qvz[e], qnxx, qnxy, J, stride, ja );
}

// ---------------------------------------------------------------------------
// Fused particle kernel: push -> move/deposit -> reflecting walls -> leaver
// detection, one CTA per (species, tile, chunk) work item.
//
//   PUSH   0 none, 1 Boris, 2 Boris with Euler-Rodrigues rotation
//   MOVE   0 none, 1 move (free streaming), 2 move + deposit
//   DETECT record leavers (bnd_check, particles.cpp:212-303)
//
// E and B tiles (guard cells included, the contiguous tile_vol block) are
// staged into shared memory with one bulk asynchronous copy each; the tile
// current is accumulated in shared memory and added to the raw current buffer
// with one bulk reduce-add.  Thread t handles particles t and t+256 of each
// 512-particle block (2 per thread keeps 4 CTAs per SM resident without
// spills, 35% faster than 4 per thread): every access is a fully coalesced 128 B
// warp transaction, and consecutive lanes (consecutive particles, which the
// injection order puts in consecutive cells) spread over the shared-memory
// banks (about 2-way conflicts; as particles drift between the cells of their
// tile the order decays towards random cells, about 3.5-way, which the
// optional in-tile reorder undoes).  Particles that stay in their cell deposit
// one segment at once; particles that cross a cell edge are queued per warp
// and split/deposited in full-warp passes, so the split runs on full warps
// (only a third segment, for the rare double crossings, diverges).
// ---------------------------------------------------------------------------
// Block-wide exclusive scan of one value per thread; the block total is
// written to *total (a shared variable) and visible on return.
template < int NT >
__device__ __forceinline__ long long block_exscan( long long v, long long * total ) {
    static_assert( NT % 32 == 0 && NT <= 1024, "block size" );
    __shared__ long long wsum[ NT / 32 ];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    long long incl = v;
#pragma unroll
    for ( int o = 1; o < 32; o <<= 1 ) {
        const long long y = __shfl_up_sync( 0xffffffffu, incl, o );
        if ( lane >= o ) incl += y;
    }
    if ( lane == 31 ) wsum[w] = incl;
    __syncthreads();
    if ( w == 0 ) {
        const long long s = ( lane < NT / 32 ) ? wsum[lane] : 0;
        long long si = s;
#pragma unroll
        for ( int o = 1; o < 32; o <<= 1 ) {
            const long long y = __shfl_up_sync( 0xffffffffu, si, o );
            if ( lane >= o ) si += y;
        }
        if ( lane < NT / 32 ) wsum[lane] = si - s;
        if ( lane == NT / 32 - 1 ) *total = si;
    }
    __syncthreads();
    const long long r = wsum[w] + incl - v;
    __syncthreads();
    return r;
}

// Target tile index along one axis for a particle leaving through v (periodic
// wrap, or -1 past an open edge).
__device__ __forceinline__ int wrap_tile( int v, int n, int periodic ) {
    if ( periodic ) { if ( v < 0 ) v += n; if ( v >= n ) v -= n; return v; }
    return ( v >= 0 && v < n ) ? v : -1;
}

constexpr int PK_THREADS = 256;
constexpr int PK_PPT = 2;                   // particles per thread per block iteration
// Particles between fixed-point flushes: at most 3 additions per particle and
// accumulator pair, 61,440 < 2^16 per group.  Tiles of 16x16 cells at 8x8
// particles per cell (16,384 on average) then run without a flush.
constexpr int FLUSH_PARTICLES = 20480;
static_assert( FLUSH_PARTICLES % ( PK_PPT * PK_THREADS ) == 0, "flush groups hold whole blocks" );

// Adds the fixed-point tile current accumulated so far (hi words at acc[0, n),
// full words at acc[n, 2n)) to the raw current of the tile and clears it.  Out
// of line: it runs once per FLUSH_PARTICLES particles of a CTA, at most.
__device__ __noinline__ void jfix_flush( int * acc, int n, float * __restrict__ dst, double inv ) {
    __syncthreads();
    unsigned int * full = reinterpret_cast<unsigned int *>( acc ) + n;
    for ( int i = threadIdx.x; i < n; i += blockDim.x ) {
        const int h = acc[i];
        const unsigned int l = full[i];
        if ( h != 0 || l != 0 ) {
            atomicAdd( dst + i, (float) jfix_value( h, l, inv ) );
            acc[i] = 0;
            full[i] = 0;
        }
    }
    __syncthreads();
}

// JT is the type of the tile current accumulated in shared memory: float
// (FP32 sums, as the reference), double (FP64 sums) or int (fixed point in
// two 32-bit words, order-independent); the last two are rounded
// to FP32 once per cell when the tile is added to the global deposit buffer.
// TN > 0 fixes square TN x TN tiles at compile time, so every shared-memory
// offset of the interpolation and deposit stencils is an immediate; TN = 0
// reads the tile shape from the run descriptor.
template < int PUSH, int MOVE, bool DETECT, typename JT = float, int TN = 0 >
__global__ void __launch_bounds__( PK_THREADS, 4 )
k_particles( const Item * __restrict__ items, const SpDev * __restrict__ sps,
             const RunDev * __restrict__ runs, const int * __restrict__ shifts )
{
    extern __shared__ __align__( 16 ) unsigned char smem_raw[];
    const Item it = items[ blockIdx.x ];
    const SpDev & S = sps[ it.sp ];
    const RunDev & R = runs[ S.run ];
    const int tv = TN ? ( ( ( TN + 3 ) * ( TN + 3 ) + 3 ) & ~3 ) : R.tile_vol;
    const int t = it.tile;
    const int nchunk = S.nchunk;

    // shared memory: [E tile][B tile][tile current (JT; fixed point: hi
    //                words then lo words)][mbarrier][energy partials][crossing queues]
    constexpr bool FIX = std::is_same<JT, int>::value;
    constexpr int JW = FIX ? 2 : 1;
    float * sE = reinterpret_cast<float *>( smem_raw );
    float * sB = sE + 3 * tv;
    JT * sJ = reinterpret_cast<JT *>( sB + 3 * tv );
    uint64_t * bar = reinterpret_cast<uint64_t *>( sJ + 3 * tv * JW );
    double * sred = reinterpret_cast<double *>( bar + 1 );
    CrossQueue * xq = reinterpret_cast<CrossQueue *>( sred + PK_THREADS / 32 );

    const int np = S.np[ t ];
    const int off = S.off[ t ];
    // CTAs in proportion to the tile's particles (balanced chunking)
    const int nc = S.chunk_target > 0 ? max( 1, min( nchunk, ( np + S.chunk_target - 1 ) / S.chunk_target ) ) : nchunk;
    const int per = ( ( np + nc - 1 ) / nc + 3 ) & ~3;
    const int begin = it.chunk < nc ? it.chunk * per : np;
    const int end = min( np, begin + per );
    const int eidx = t * nchunk + it.chunk;

    if ( begin >= end ) {
        if ( PUSH && threadIdx.x == 0 ) S.energy[ eidx ] = 0.0;
        return;
    }
    // leavers per direction (bnd_check's per-direction counts), added to the
    // tile's counts once per CTA
    __shared__ int s_dir[9];
    if ( DETECT && threadIdx.x < 9 ) s_dir[ threadIdx.x ] = 0;

    if ( PUSH ) {
        if ( threadIdx.x == 0 ) {
            mbar_init( bar, 1 );
            fence_mbar_init();
        }
        __syncthreads();
        if ( threadIdx.x == 0 ) {
            const uint32_t bytes = 12u * tv;
            mbar_arrive_expect_tx( bar, 2 * bytes );
            bulk_g2s( sE, R.E + (size_t) t * 3 * tv, bytes, bar );
            bulk_g2s( sB, R.B + (size_t) t * 3 * tv, bytes, bar );
        }
    }
    if ( MOVE == 2 ) {
        for ( int i = threadIdx.x; i < 3 * tv * JW; i += blockDim.x ) sJ[i] = (JT) 0;
    }
    if ( PUSH ) {
        // an expired wait: the item's particles, current and energy are left
        // as they were (the step is reported failed)
        if ( bulk_wait_or_abandon( bar, R.status, R.wait_limit ) ) {
            if ( threadIdx.x == 0 ) S.energy[ eidx ] = 0.0;
            return;
        }
    } else {
        __syncthreads();
    }

    const int ys = TN ? TN + 3 : R.extx;
    const int gc_off = TN ? TN + 4 : R.gc_off;
    const float * Ec = sE + 3 * gc_off;
    const float * Bc = sB + 3 * gc_off;
    JT * Jc = sJ + 3 * gc_off;
    const int nxx = TN ? TN : R.nxx, nxy = TN ? TN : R.nxy;
    const int tx = t % R.ntx, ty = t / R.ntx;
    const int shift = ( MOVE && shifts ) ? shifts[ it.sp ] : 0;
    const bool euler = ( PUSH == 2 );

    // reflecting walls handled here (species.cpp:1854-1989): lower rule on the
    // first tile column, upper rule on the last one; x first, then y.
    const int rxl = ( MOVE && tx == 0 && ( S.bc[0] > 1 || S.bc[1] > 1 ) && S.bc[0] == 2 );
    const int rxu = ( MOVE && tx != 0 && tx == R.ntx - 1 && ( S.bc[0] > 1 || S.bc[1] > 1 ) && S.bc[1] == 2 );
    const int ryl = ( MOVE && ty == 0 && ( S.bc[2] > 1 || S.bc[3] > 1 ) && S.bc[2] == 2 );
    const int ryu = ( MOVE && ty != 0 && ty == R.nty - 1 && ( S.bc[2] > 1 || S.bc[3] > 1 ) && S.bc[3] == 2 );
    const bool walls = ( rxl | rxu | ryl | ryu ) != 0;

    const float alpha = S.alpha;
    // current factors: half of q dx / dt, and q / 2 (for q vz / 2), times the
    // fixed-point scale (exact power-of-two products)
    const float jsf = FIX ? S.jscale : 1.0f;
    const float dt_dx = S.dt_dx, dt_dy = S.dt_dy, qhalf = 0.5f * S.q * jsf;
    const float qnxx = 0.5f * S.qnx * jsf, qnxy = 0.5f * S.qny * jsf;
    const JAcc ja = { S.jscale, 3 * tv };

    uint32_t * __restrict__ pc = S.A.cell + off;
    float * __restrict__ pxx = S.A.xx + off;
    float * __restrict__ pxy = S.A.xy + off;
    float * __restrict__ pux = S.A.ux + off;
    float * __restrict__ puy = S.A.uy + off;
    float * __restrict__ puz = S.A.uz + off;

    double energy = 0.0;
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = ( 1u << lane ) - 1u;
    CrossQueue & Q = xq[ threadIdx.x >> 5 ];
    int qh = 0, qt = 0;                         // warp-uniform ring head / tail

    // Groups of FLUSH_PARTICLES: with the fixed-point tile current the
    // accumulators are flushed between groups (at most 3 additions per
    // particle and entry, well below the 2^16 the words can take).
    for ( int g0 = begin; g0 < end; g0 += FLUSH_PARTICLES ) {
        if constexpr ( FIX && MOVE == 2 ) {
            if ( g0 != begin ) jfix_flush( reinterpret_cast<int *>( sJ ), 3 * tv, R.Jdep + (size_t) t * 3 * tv, S.jscale_inv );
        }
        const int gend = min( end, g0 + FLUSH_PARTICLES );
        for ( int b0 = g0; b0 < gend; b0 += PK_PPT * PK_THREADS ) {
            uint32_t c[PK_PPT] = {}; float x0[PK_PPT], x1[PK_PPT], u0[PK_PPT], u1[PK_PPT], u2[PK_PPT];
            int leave_dir[PK_PPT];
#pragma unroll
            for ( int k = 0; k < PK_PPT; k++ ) {
                const int i = b0 + k * PK_THREADS + threadIdx.x;
                if ( i < end ) {
                    c[k] = pc[i]; x0[k] = pxx[i]; x1[k] = pxy[i];
                    if ( PUSH || MOVE ) { u0[k] = pux[i]; u1[k] = puy[i]; u2[k] = puz[i]; }
                }
            }
#pragma unroll
            for ( int k = 0; k < PK_PPT; k++ ) {
                const int i = b0 + k * PK_THREADS + threadIdx.x;
                bool valid = i < end;
                bool cross = false;
                leave_dir[k] = 4;
                int ix = 0, iy = 0, oix = 0, oiy = 0;
                float d0 = 0.f, d1 = 0.f, qz = 0.f, ox = 0.f, oy = 0.f;
                if ( PUSH || MOVE ) {
                    ix = cell_x( c[k] ); iy = cell_y( c[k] );
                    // Sorted particles sit inside their tile; anything else (only
                    // reachable by moving twice without a sort) is flagged and left
                    // untouched so no field or current access leaves the tile block.
                    // TN x TN tiles (TN a power of two): both 16-bit cell
                    // coordinates inside [0, TN) exactly when no bit above TN - 1 is set
                    const bool bad = valid && ( ( TN > 0 && ( TN & ( TN - 1 ) ) == 0 )
                                   ? ( c[k] & ~( (uint32_t) ( TN - 1 ) * 0x10001u ) ) != 0
                                   : ( ix < 0 || ix >= nxx || iy < 0 || iy >= nxy ) );
                    const unsigned mbad = __ballot_sync( 0xffffffffu, bad );
                    if ( mbad ) {
                        if ( lane == __ffs( mbad ) - 1 ) atomicOr( R.status, ST_BAD_CELL );
                        valid = valid && !bad;
                    }
                } else if ( valid ) {
                    ix = cell_x( c[k] ); iy = cell_y( c[k] );
                }
                if ( valid ) {
                    if ( PUSH ) {
                        float ex, ey, ez, bx, by, bz;
                        interpolate_fld( Ec, Bc, ys, ix, iy, x0[k], x1[k], ex, ey, ez, bx, by, bz );
                        if ( euler ) dudt_boris_euler( alpha, ex, ey, ez, bx, by, bz, u0[k], u1[k], u2[k], energy );
                        else         dudt_boris( alpha, ex, ey, ez, bx, by, bz, u0[k], u1[k], u2[k], energy );
                    }
                    if ( MOVE ) {
                        // species.cpp:1431-1489
                        const float rg = rgamma( u0[k], u1[k], u2[k] );
                        d0 = dt_dx * rg * u0[k];
                        d1 = dt_dy * rg * u1[k];
                        const float x1x = x0[k] + d0, x1y = x1[k] + d1;
                        const int dix = ( ( x1x >= 0.5f ) - ( x1x < -0.5f ) );
                        const int diy = ( ( x1y >= 0.5f ) - ( x1y < -0.5f ) );
                        if ( MOVE == 2 ) {
                            qz = qhalf * u2[k] * rg;
                            cross = ( dix | diy ) != 0;
                            if ( !cross )
                                dep_current_seg( ix, iy, x0[k], x1[k], x1x, x1y, qnxx, qnxy, qz, Jc, ys, ja );
                        }
                        ox = x0[k]; oy = x1[k]; oix = ix; oiy = iy;
                        x0[k] = x1x - dix; x1[k] = x1y - diy;
                        ix += dix + shift; iy += diy;
                        if ( walls ) {
                            if ( rxl && ix < 0 )    { ix += 1; x0[k] = -x0[k]; u0[k] = -u0[k]; }
                            if ( rxu && ix >= nxx ) { ix -= 1; x0[k] = -x0[k]; u0[k] = -u0[k]; }
                            if ( ryl && iy < 0 )    { iy += 1; x1[k] = -x1[k]; u1[k] = -u1[k]; }
                            if ( ryu && iy >= nxy ) { iy -= 1; x1[k] = -x1[k]; u1[k] = -u1[k]; }
                        }
                        c[k] = pack_cell( ix, iy );
                    }
                    if ( DETECT ) {
                        const int xcross = ( ix >= nxx ) - ( ix < 0 );
                        const int ycross = ( iy >= nxy ) - ( iy < 0 );
                        leave_dir[k] = ( ycross + 1 ) * 3 + ( xcross + 1 );
                    }
                }
                if ( MOVE == 2 ) {
                    // queue cell-crossing particles (warp-uniform point)
                    const unsigned m = __ballot_sync( 0xffffffffu, cross );
                    if ( m ) {
                        if ( cross ) {
                            const int e = ( qt + __popc( m & lt_mask ) ) & ( XQ - 1 );
                            Q.cell[e] = pack_cell( oix, oiy );
                            Q.x0x[e] = ox; Q.x0y[e] = oy;
                            Q.dx[e] = d0; Q.dy[e] = d1; Q.qvz[e] = qz;
                        }
                        qt += __popc( m );
                        if ( qt - qh >= 32 ) {
                            __syncwarp();
                            drain_entry( Q, ( qh + lane ) & ( XQ - 1 ), qnxx, qnxy, Jc, ys, ja );
                            qh += 32;
                            __syncwarp();
                        }
                    }
                }
            }
#pragma unroll
            for ( int k = 0; k < PK_PPT; k++ ) {
                const int i = b0 + k * PK_THREADS + threadIdx.x;
                if ( i < end ) {
                    if ( MOVE ) { pc[i] = c[k]; pxx[i] = x0[k]; pxy[i] = x1[k]; }
                    if ( PUSH || rxl || rxu ) pux[i] = u0[k];
                    if ( PUSH || ryl || ryu ) puy[i] = u1[k];
                    if ( PUSH ) puz[i] = u2[k];
                }
            }

            if ( DETECT ) {
                // warp-aggregated append of leaver indices (one global atomic per warp)
                int nl = 0;
#pragma unroll
                for ( int k = 0; k < PK_PPT; k++ ) nl += ( leave_dir[k] != 4 );
                const unsigned any = __ballot_sync( 0xffffffffu, nl > 0 );
                if ( any ) {
                    int incl = nl;
#pragma unroll
                    for ( int o = 1; o < 32; o <<= 1 ) {
                        const int v = __shfl_up_sync( 0xffffffffu, incl, o );
                        if ( lane >= o ) incl += v;
                    }
                    const int total = __shfl_sync( 0xffffffffu, incl, 31 );
                    int wbase = 0;
                    if ( lane == 31 ) wbase = atomicAdd( S.nidx + t, total );
                    wbase = __shfl_sync( 0xffffffffu, wbase, 31 );
                    int pos = wbase + incl - nl;
#pragma unroll
                    for ( int k = 0; k < PK_PPT; k++ ) {
                        if ( leave_dir[k] != 4 ) {
                            const int li = b0 + k * PK_THREADS + threadIdx.x;
                            S.idx[ off + pos ] = li;
                            // leaver outbox in buffer B (unused outside a repack),
                            // so that the sort reads the leavers coalesced
                            const size_t o = (size_t) off + pos;
                            S.B.cell[o] = c[k]; S.B.xx[o] = x0[k]; S.B.xy[o] = x1[k];
                            if ( PUSH || MOVE ) { S.B.ux[o] = u0[k]; S.B.uy[o] = u1[k]; S.B.uz[o] = u2[k]; }
                            else { S.B.ux[o] = pux[li]; S.B.uy[o] = puy[li]; S.B.uz[o] = puz[li]; }
                            pos++;
                            // counted per direction when the target tile exists
                            const int ttx = wrap_tile( tx + leave_dir[k] % 3 - 1, R.ntx, S.perx );
                            const int tty = wrap_tile( ty + leave_dir[k] / 3 - 1, R.nty, S.pery );
                            if ( ttx >= 0 && tty >= 0 ) atomicAdd( &s_dir[ leave_dir[k] ], 1 );
                        }
                    }
                }
            }
        }
    }
    if ( MOVE == 2 && qt != qh ) {
        __syncwarp();
        if ( lane < qt - qh ) drain_entry( Q, ( qh + lane ) & ( XQ - 1 ), qnxx, qnxy, Jc, ys, ja );
    }

    if ( PUSH ) {
        // deterministic per-item energy: warp tree, then warps in order
#pragma unroll
        for ( int o = 16; o > 0; o >>= 1 ) energy += __shfl_down_sync( 0xffffffffu, energy, o );
        if ( lane == 0 ) sred[ threadIdx.x >> 5 ] = energy;
    }
    __syncthreads();
    const float * sJout = reinterpret_cast<const float *>( sJ );
    if ( MOVE == 2 && !std::is_same<JT, float>::value ) {
        // round the FP64 or fixed-point tile current once per cell, into the E tile's place
        for ( int i = threadIdx.x; i < 3 * tv; i += blockDim.x ) {
            if constexpr ( FIX )
                sE[i] = (float) jfix_value( sJ[i], reinterpret_cast<const unsigned int *>( sJ )[ 3 * tv + i ],
                                            S.jscale_inv );
            else sE[i] = (float) sJ[i];
        }
        sJout = sE;
        __syncthreads();
    }
    if ( DETECT && threadIdx.x < 9 && threadIdx.x != 4 ) {
        const int v = s_dir[ threadIdx.x ];
        if ( v ) atomicAdd( S.cnt + 9 * t + threadIdx.x, v );
    }
    if ( threadIdx.x == 0 ) {
        if ( PUSH ) {
            double e = 0.0;
            for ( int w = 0; w < ( (int) blockDim.x >> 5 ); w++ ) e += sred[w];
            S.energy[ eidx ] = e;
        }
        if ( MOVE && it.chunk == 0 ) atomicAdd( S.nmove, (unsigned long long) np );
        if ( MOVE == 2 ) {
            fence_proxy_async_smem();
            bulk_s2g_add_f32( R.Jdep + (size_t) t * 3 * tv, sJout, 12u * tv );
            bulk_commit();
            // the CTA may leave once its shared memory has been read; the
            // global additions complete before the kernel does
            bulk_wait_read_all();
        }
    }
}

// ---------------------------------------------------------------------------
// Tile sort (particles.cpp:212-614 semantics: afterwards every particle sits
// in the slot of the tile that holds its cell, at positions [0, np) of that
// slot; the per-tile multiset is what the reference fixes, its order within
// the tile depends on thread timing there as here).
//
// The particle kernel leaves, per tile t: the leavers' payload in the outbox
// (buffer B at off[t] + k, k < nidx[t]), their slot indices (idx at
// off[t] + k) and the number leaving in each direction d (cnt[9 t + d],
// d = 3 (ycross + 1) + xcross + 1, 4 meaning "stays").  Then:
//   k_sort_check   per tile: incoming per direction from the 8 neighbour
//                  counts, their offsets (base), the new count, and whether
//                  it fits the tile's slot;
//   k_sort_plan    per species: in place (mode 0) if every tile fits, else
//                  a new slot layout (mode 1, a repack through buffer B);
//   k_sort_local   per tile: the slots that are empty below the new count
//                  (leavers' slots, or room after the old count) are listed;
//                  stayers above the new count move into the first of them,
//                  the rest are for the incoming particles;
//   k_sort_scatter per source tile: each leaver goes from the outbox
//                  straight to its slot in the target tile, at rank
//                  base(target, direction) + its rank among this tile's
//                  leavers in that direction -- no staging copy and no
//                  returning global atomics.
// ---------------------------------------------------------------------------

// Tile reached from tile t through direction d (wrap or -1 past an open edge).
__device__ __forceinline__ int neighbor_tile( int t, int d, int ntx, int nty, int perx, int pery ) {
    const int wx = wrap_tile( t % ntx + d % 3 - 1, ntx, perx );
    const int wy = wrap_tile( t / ntx + d / 3 - 1, nty, pery );
    return ( wx >= 0 && wy >= 0 ) ? wy * ntx + wx : -1;
}

constexpr int CHECK_THREADS = 256;

// One thread per (species, tile) item.  Particles arriving at t through
// direction d come from the neighbour in the opposite direction 8 - d.
__global__ void __launch_bounds__( CHECK_THREADS )
k_sort_check( const Item * __restrict__ items, int nitems, const SpDev * __restrict__ sps,
              const RunDev * __restrict__ runs, int use_extra, int * __restrict__ rlist )
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if ( i == 0 ) rlist[0] = 0;                   // the plan lists the species that repack
    if ( i >= nitems ) return;
    const Item it = items[i];
    const SpDev & S = sps[ it.sp ];
    const RunDev & R = runs[ S.run ];
    const int t = it.tile;
    int g[9];
#pragma unroll
    for ( int d = 0; d < 9; d++ ) {
        const int src = d == 4 ? -1 : neighbor_tile( t, 8 - d, R.ntx, R.nty, S.perx, S.pery );
        g[d] = src >= 0 ? S.cnt[ 9 * src + d ] : 0;
    }
    int in = 0;
#pragma unroll
    for ( int d = 0; d < 9; d++ ) { S.base[ 9 * t + d ] = in; in += g[d]; }
    const int stay = S.np[t] - S.nidx[t];
    const int ex = ( use_extra && S.extra ) ? S.extra[t] : 0;
    S.in_cnt[t] = in;
    S.new_np[t] = stay + in;
    int rel = 0;
    if ( stay + in + ex > S.cap[t] ) {
        // a new slot in the pool, with room to grow (reloc_room times its
        // count, at least twice the minimum slack): a tile that outgrew its
        // slot is usually still growing
        rel = 1;
        atomicAdd( S.nmove + 2, 1ull );
        const int grow = max( 2 * S.min_slack, (int) ( S.reloc_room * ( stay + in ) ) );
        S.new_cap[t] = ( ( stay + in + ex + 3 ) & ~3 ) + ( ( grow + 3 ) & ~3 );
        atomicOr( S.overflow, 1 );
    }
    S.reloc[t] = rel;
}

constexpr int PLAN_THREADS = 1024;
// rlist entries: species index, with this bit set for a species that only
// relocates tiles (mode 3) rather than repacking (mode 1)
constexpr int RLIST_RELOCATE = 1 << 30;

// One CTA per species.  In place (mode 0) unless a tile overflowed its slot;
// then the repack layout (mode 1): need[t] = new count + injection reserve,
// rounded up to 4, and the free capacity spread in proportion to
// need + min_slack (multiples of 4); mode 2 when the buffer cannot hold the
// new total (ST_CAPACITY: the host grows buffers before that can happen).
__global__ void __launch_bounds__( PLAN_THREADS )
k_sort_plan( const SpDev * __restrict__ sps, const int * __restrict__ species_list,
             const RunDev * __restrict__ runs, int use_extra, int * __restrict__ rlist )
{
    const SpDev & S = sps[ species_list[ blockIdx.x ] ];
    const RunDev & R = runs[ S.run ];
    const int over = *S.overflow;
    __syncthreads();

    if ( !over ) {
        if ( threadIdx.x == 0 ) *S.mode = 0;
        return;
    }
    if ( threadIdx.x == 0 ) *S.overflow = 0;
    const int nt = S.ntiles;
    const int per = ( nt + PLAN_THREADS - 1 ) / PLAN_THREADS;
    const int t0 = min( nt, (int) threadIdx.x * per ), t1 = min( nt, t0 + per );
    __shared__ long long s_total;
    // relocation (mode 3): the tiles that outgrew their slots get new slots
    // from the pool, everything else sorts in place; a repack only when the
    // pool cannot hold them
    {
        long long rsum = 0, rn = 0, rp = 0;
        for ( int t = t0; t < t1; t++ )
            if ( S.reloc[t] ) { rsum += S.new_cap[t]; rn += 1; rp += S.np[t]; }
        long long ro = block_exscan< PLAN_THREADS >( rsum, &s_total );
        const long long rtotal = s_total;
        const long long pool = *S.pool;
        if ( pool + rtotal <= (long long) S.max_part ) {
            // new slots, and the list of the relocated tiles with the packed
            // start of their particles (the local kernel's grid-stride copy)
            long long ri = block_exscan< PLAN_THREADS >( rn, &s_total );
            const long long nrel = s_total;
            long long rs = block_exscan< PLAN_THREADS >( rp, &s_total );
            const long long ptotal = s_total;
            ro += pool;
            for ( int t = t0; t < t1; t++ )
                if ( S.reloc[t] ) {
                    S.new_off[t] = (int) ro; ro += S.new_cap[t];
                    S.rel_tile[ri] = t; S.rel_start[ri] = (int) rs; ri += 1; rs += S.np[t];
                    S.hs[t] = S.np[t] - S.nidx[t];  // the stayers, then the incoming
                    S.stage_cnt[t] = 0;
                }
            __syncthreads();                      // every thread has read the pool start
            if ( threadIdx.x == 0 ) {
                *S.pool = (int) ( pool + rtotal ); *S.mode = 3;
                S.rel_start[ nrel ] = (int) ptotal; *S.rel_n = (int) nrel;
                rlist[ 1 + atomicAdd( rlist, 1 ) ] = species_list[ blockIdx.x ] | RLIST_RELOCATE;
            }
            return;
        }
        __syncthreads();
    }
    long long need_sum = 0, w_sum = 0, np_sum = 0;
    for ( int t = t0; t < t1; t++ ) {
        const int ex = ( use_extra && S.extra ) ? S.extra[t] : 0;
        const int need = ( S.new_np[t] + ex + 3 ) & ~3;
        need_sum += need;
        w_sum += need + S.min_slack;
        np_sum += S.np[t];
        S.stage_cnt[t] = 0;
    }
    // packed position of each tile's first particle (the repack's index space)
    long long pk = block_exscan< PLAN_THREADS >( np_sum, &s_total );
    for ( int t = t0; t < t1; t++ ) { S.hs[t] = (int) pk; pk += S.np[t]; }
    __syncthreads();
    block_exscan< PLAN_THREADS >( need_sum, &s_total );
    const long long need_total = s_total;
    __syncthreads();
    block_exscan< PLAN_THREADS >( w_sum, &s_total );
    const long long w_total = s_total;
    const long long free_cap = (long long) S.max_part - need_total;
    if ( free_cap < 0 ) {
        if ( threadIdx.x == 0 ) { *S.mode = 2; atomicOr( R.status, ST_CAPACITY ); }
        return;
    }
    // the free capacity: slack in the slots, a share (pool_frac) left as the pool
    const long long spread = (long long) ( (double) free_cap * ( 1.0 - S.pool_frac ) );
    long long cap_sum = 0;
    for ( int t = t0; t < t1; t++ ) {
        const int ex = ( use_extra && S.extra ) ? S.extra[t] : 0;
        const int need = ( S.new_np[t] + ex + 3 ) & ~3;
        const long long slack = w_total > 0 ? ( spread * ( need + S.min_slack ) ) / w_total : 0;
        const int c = need + (int) ( slack & ~3LL );
        S.new_cap[t] = c;
        cap_sum += c;
    }
    __syncthreads();
    long long pc = block_exscan< PLAN_THREADS >( cap_sum, &s_total );
    for ( int t = t0; t < t1; t++ ) { S.new_off[t] = (int) pc; pc += S.new_cap[t]; }
    if ( threadIdx.x == 0 ) {
        *S.pool = (int) s_total;
        *S.mode = 1;
        S.nmove[1] += 1;
        rlist[ 1 + atomicAdd( rlist, 1 ) ] = species_list[ blockIdx.x ];
    }
}

__device__ __forceinline__ void copy_particle( const PartArrays & d, size_t di, const PartArrays & s, size_t si ) {
    d.cell[di] = s.cell[si]; d.xx[di] = s.xx[si]; d.xy[di] = s.xy[si];
    d.ux[di] = s.ux[si]; d.uy[di] = s.uy[si]; d.uz[di] = s.uz[si];
}

constexpr int SORT_THREADS = 256;
constexpr int SORT_WARPS = SORT_THREADS / 32;
constexpr int SU = 4;                             // sort entries per lane in flight

// Repack, first half (mode 1): every particle of the species goes to buffer B
// in the new slot layout -- stayers into their own tile's new slot, leavers
// into their target's.  The whole grid strides over the species' particles
// in packed order (q-th particle: tile t with hs[t] <= q < hs[t] + np[t], the
// packed offsets the plan wrote into hs), so a tile's particles are spread
// over all CTAs however unevenly the tiles are filled, and slack is not
// visited; slots are claimed per destination with one atomic per group of
// lanes sharing it.
__device__ __noinline__ void repack_out( const SpDev & S, const RunDev & R ) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = ( 1u << lane ) - 1u;
    const int nt = S.ntiles, ntx = R.ntx, nty = R.nty, nxx = R.nxx, nxy = R.nxy;
    const long long n = (long long) S.hs[ nt - 1 ] + S.np[ nt - 1 ];
    for ( long long q0 = (long long) blockIdx.x * blockDim.x; q0 < n; q0 += (long long) gridDim.x * blockDim.x ) {
        const long long q = q0 + threadIdx.x;
        int dest = -1, ix = 0, iy = 0, xc = 0, yc = 0;
        long long p = 0;
        if ( q < n ) {
            // the last tile whose first packed position is at or before q (a
            // tile without particles shares its position with the next one)
            int lo = 0, hi = nt - 1;
            while ( lo < hi ) {
                const int mid = ( lo + hi + 1 ) >> 1;
                if ( S.hs[mid] <= q ) lo = mid; else hi = mid - 1;
            }
            const int t = lo, i = (int) ( q - S.hs[t] );
            p = (long long) S.off[t] + i;
            if ( i >= 0 && i < S.np[t] ) {
                const uint32_t c = S.A.cell[p];
                ix = cell_x( c ); iy = cell_y( c );
                xc = ( ix >= nxx ) - ( ix < 0 ); yc = ( iy >= nxy ) - ( iy < 0 );
                const int ttx = wrap_tile( t % ntx + xc, ntx, S.perx ), tty = wrap_tile( t / ntx + yc, nty, S.pery );
                dest = ( ttx >= 0 && tty >= 0 ) ? tty * ntx + ttx : -1;
            }
        }
        const unsigned same = __match_any_sync( 0xffffffffu, dest );
        const int leader = __ffs( same ) - 1;
        int base = 0;
        if ( dest >= 0 && lane == leader ) base = atomicAdd( S.stage_cnt + dest, __popc( same ) );
        base = __shfl_sync( same, base, leader );
        if ( dest >= 0 ) {
            const size_t d = (size_t) S.new_off[dest] + base + __popc( same & lt );
            copy_particle( S.B, d, S.A, (size_t) p );
            if ( xc != 0 || yc != 0 ) S.B.cell[d] = pack_cell( ix - xc * nxx, iy - yc * nxy );
        }
    }
}

// Relocation (mode 3): the stayers of every tile that outgrew its slot are
// copied into its new slot from the pool.  The whole grid strides over those
// tiles' particles in packed order (rel_start, written by the plan), so a big
// tile is spread over all CTAs; places in the new slot are claimed per tile
// with one atomic per group of lanes in the same tile.
__device__ __noinline__ void relocate_out( const SpDev & S, const RunDev & R ) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = ( 1u << lane ) - 1u;
    const int nrel = *S.rel_n, nxx = R.nxx, nxy = R.nxy;
    if ( nrel <= 0 ) return;
    const long long n = S.rel_start[ nrel ];
    for ( long long q0 = (long long) blockIdx.x * blockDim.x; q0 < n; q0 += (long long) gridDim.x * blockDim.x ) {
        const long long q = q0 + threadIdx.x;
        int t = -1;
        long long p = 0;
        if ( q < n ) {
            int lo = 0, hi = nrel - 1;
            while ( lo < hi ) {
                const int mid = ( lo + hi + 1 ) >> 1;
                if ( S.rel_start[mid] <= q ) lo = mid; else hi = mid - 1;
            }
            const int tt = S.rel_tile[lo];
            p = (long long) S.off[tt] + ( q - S.rel_start[lo] );
            const uint32_t c = S.A.cell[p];
            const int ix = cell_x( c ), iy = cell_y( c );
            if ( ix >= 0 && ix < nxx && iy >= 0 && iy < nxy ) t = tt;    // leavers are in the outbox
        }
        const unsigned same = __match_any_sync( 0xffffffffu, t );
        const int leader = __ffs( same ) - 1;
        int base = 0;
        if ( t >= 0 && lane == leader ) base = atomicAdd( S.stage_cnt + t, __popc( same ) );
        base = __shfl_sync( same, base, leader );
        if ( t >= 0 ) copy_particle( S.A, (size_t) S.new_off[t] + base + __popc( same & lt ), S.A, (size_t) p );
    }
}

// Repack, second half: B -> A over the whole buffer (slack included),
// 16-byte vectors (the arrays are cudaMalloc'd, 256-byte aligned); the last
// max_part % 4 entries are copied singly.  A sweep of the whole buffer in
// vectors is faster than visiting only the new layout's particles, which
// needs a search for each one's tile.
__device__ __forceinline__ void copy_vec( void * dst, const void * src, long long i ) {
    reinterpret_cast<uint4 *>( dst )[i] = reinterpret_cast<const uint4 *>( src )[i];
}

__device__ __noinline__ void repack_in( const SpDev & S ) {
    const long long n = S.max_part, n4 = n / 4;
    const long long stride = (long long) gridDim.x * blockDim.x;
    for ( long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride ) {
        copy_vec( S.A.cell, S.B.cell, i ); copy_vec( S.A.xx, S.B.xx, i ); copy_vec( S.A.xy, S.B.xy, i );
        copy_vec( S.A.ux, S.B.ux, i );     copy_vec( S.A.uy, S.B.uy, i ); copy_vec( S.A.uz, S.B.uz, i );
    }
    for ( long long p = 4 * n4 + blockIdx.x * (long long) blockDim.x + threadIdx.x; p < n; p += stride )
        copy_particle( S.A, (size_t) p, S.B, (size_t) p );
}

// Per tile (WPT warps per tile; 1 when there are many tiles, a whole CTA when
// there are few and they are large): with nn = np - nidx + in the new count,
// list the slots that will be empty below nn -- the leavers' slots below nn
// (aux, appended through a per-tile shared counter from warp ballots), then
// np .. nn-1 when the tile grows -- and the stayers at or above nn (aux2).
// Stayer q moves into empty slot q; the remaining entries, from hs = number of
// such stayers on, receive the incoming particles (k_sort_scatter).  Also
// clears the tile's direction counts for the next step (k_sort_check has read
// them).  Species in mode 1 are repacked instead (first half).
template < int WPT >
__global__ void __launch_bounds__( SORT_THREADS )
k_sort_local( const Item * __restrict__ items, int nitems, const SpDev * __restrict__ sps,
              const int * __restrict__ rlist, const RunDev * __restrict__ runs )
{
    constexpr int TPB = SORT_WARPS / WPT;         // tiles per CTA
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tib = warp / WPT, sub = warp % WPT;
    const unsigned lt = ( 1u << lane ) - 1u;
    __shared__ int s_ne[TPB], s_ns[TPB];
    if ( sub == 0 && lane == 0 ) { s_ne[tib] = 0; s_ns[tib] = 0; }
    if ( WPT > 1 ) __syncthreads(); else __syncwarp();

    const int wi = blockIdx.x * TPB + tib;
    bool active = wi < nitems, rel = false;
    Item it{};
    const SpDev * Sp = nullptr;
    if ( active ) {
        it = items[ wi ];
        Sp = &sps[ it.sp ];
        if ( sub == 0 && lane < 9 ) Sp->cnt[ 9 * it.tile + lane ] = 0;
        const int mode = *Sp->mode;
        active = mode == 0 || mode == 3;
        rel = active && mode == 3 && Sp->reloc[ it.tile ];
    }
    int t = 0, np = 0, nl = 0, nn = 0, off = 0, nxx = 1, nxy = 1;
    if ( active ) {
        const SpDev & S = *Sp;
        const RunDev & R = runs[ S.run ];
        t = it.tile; nxx = R.nxx; nxy = R.nxy;
        np = S.np[t]; nl = S.nidx[t]; off = S.off[t];
        nn = np - nl + S.in_cnt[t];
    }
    if ( active && !rel ) {
        const SpDev & S = *Sp;
        // leavers' slots below nn, SU per lane in flight
        for ( int k0 = sub * 32 * SU; k0 < nl; k0 += WPT * 32 * SU ) {
            int i[SU];
#pragma unroll
            for ( int u = 0; u < SU; u++ ) {
                const int k = k0 + u * 32 + lane;
                i[u] = k < nl ? S.idx[ off + k ] : nn;
            }
#pragma unroll
            for ( int u = 0; u < SU; u++ ) {
                const bool e = i[u] < nn;
                const unsigned m = __ballot_sync( 0xffffffffu, e );
                int b = 0;
                if ( lane == 0 && m ) b = atomicAdd( &s_ne[tib], __popc( m ) );
                b = __shfl_sync( 0xffffffffu, b, 0 );
                if ( e ) S.aux[ off + b + __popc( m & lt ) ] = i[u];
            }
        }
        // stayers at or above nn
        for ( int c0 = nn + sub * 32 * SU; c0 < np; c0 += WPT * 32 * SU ) {
            uint32_t c[SU];
#pragma unroll
            for ( int u = 0; u < SU; u++ ) {
                const int ci = c0 + u * 32 + lane;
                c[u] = ci < np ? S.A.cell[ (size_t) off + ci ] : 0x80008000u;   // (-32768, -32768): outside
            }
#pragma unroll
            for ( int u = 0; u < SU; u++ ) {
                const int ix = cell_x( c[u] ), iy = cell_y( c[u] );
                const bool stay = ix >= 0 && ix < nxx && iy >= 0 && iy < nxy;
                const unsigned m = __ballot_sync( 0xffffffffu, stay );
                int b = 0;
                if ( lane == 0 && m ) b = atomicAdd( &s_ns[tib], __popc( m ) );
                b = __shfl_sync( 0xffffffffu, b, 0 );
                if ( stay ) S.aux2[ off + b + __popc( m & lt ) ] = c0 + u * 32 + lane;
            }
        }
    }
    if ( WPT > 1 ) __syncthreads(); else __syncwarp();
    // a tile that outgrew its slot: its stayers are copied by the whole grid
    // below (relocate_out); the incoming follow them in the new slot
    if ( rel ) active = false;
    if ( active ) {
        const SpDev & S = *Sp;
        const int ne = s_ne[tib], ns = s_ns[tib];
        // every empty slot below nn receives one particle: a stayer from above
        // nn or an incoming one (inconsistent counts are reported and the
        // tile's lists are not used)
        if ( ne + max( 0, nn - np ) != ns + S.in_cnt[t] ) {
            if ( sub == 0 && lane == 0 ) { S.hs[t] = nn; atomicOr( runs[ S.run ].status, ST_BAD_CELL ); }
            active = false;
        }
    }
    if ( active ) {
        const SpDev & S = *Sp;
        const int ne = s_ne[tib], ns = s_ns[tib];
        // the room after the old count, when the tile grows
        for ( int j = sub * 32 + lane; j < nn - np; j += WPT * 32 ) S.aux[ off + ne + j ] = np + j;
        // stayers above nn into the first empty slots (pairs by list rank)
        for ( int r0 = sub * 32 * SU; r0 < ns; r0 += WPT * 32 * SU ) {
            int h[SU], src[SU];
#pragma unroll
            for ( int u = 0; u < SU; u++ ) {
                const int r = r0 + u * 32 + lane;
                h[u] = r < ns ? S.aux[ off + r ] : -1;
                src[u] = r < ns ? S.aux2[ off + r ] : -1;
            }
#pragma unroll
            for ( int u = 0; u < SU; u++ )
                if ( h[u] >= 0 ) copy_particle( S.A, (size_t) off + h[u], S.A, (size_t) off + src[u] );
        }
        if ( sub == 0 && lane == 0 ) S.hs[t] = ns;
    }
    const int nr = rlist[0];
    for ( int k = 0; k < nr; k++ ) {
        const int e = rlist[ 1 + k ];
        const SpDev & S = sps[ e & ~RLIST_RELOCATE ];
        if ( e & RLIST_RELOCATE ) relocate_out( S, runs[ S.run ] );
        else repack_out( S, runs[ S.run ] );
    }
}

// Per source tile (WPT warps per tile): each leaver of the outbox goes to
// slot aux[off[tt] + hs[tt] + base[tt][d] + rank] of its target tt, rank
// counted per direction d in outbox order (shared counters, one atomic per
// group of lanes with the same direction).  Then the tile's count becomes the
// new one.  Species in mode 1 get their new slot layout and the second half
// of the repack.
template < int WPT >
__global__ void __launch_bounds__( SORT_THREADS )
k_sort_scatter( const Item * __restrict__ items, int nitems, const SpDev * __restrict__ sps,
                const int * __restrict__ rlist, const RunDev * __restrict__ runs )
{
    constexpr int TPB = SORT_WARPS / WPT;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tib = warp / WPT, sub = warp % WPT;
    const unsigned lt = ( 1u << lane ) - 1u;
    __shared__ int s_rank[TPB][9];
    __shared__ int s_off[TPB][9];                 // off[tt] of the target through direction d
    __shared__ int s_aux[TPB][9];                 // its list position of the first slot for d (-1: dropped)
    __shared__ int s_cap[TPB][9];                 // new count of the target (bound of its list and slots)
    __shared__ int s_dir[TPB][9];                 // 1: relocated target, positions without the list

    const int wi = blockIdx.x * TPB + tib;
    bool active = wi < nitems;
    Item it{};
    const SpDev * Sp = nullptr;
    int mode = -1;
    if ( active ) {
        it = items[ wi ];
        Sp = &sps[ it.sp ];
        mode = *Sp->mode;
        active = mode == 0 || mode == 3;
    }
    if ( active && sub == 0 && lane < 9 ) {
        const SpDev & S = *Sp;
        const RunDev & R = runs[ S.run ];
        const int tt = lane == 4 ? -1 : neighbor_tile( it.tile, lane, R.ntx, R.nty, S.perx, S.pery );
        int o = 0, a = -1, nn = 0, dr = 0;
        if ( tt >= 0 ) {
            // a relocated target takes its incoming right after its stayers in
            // its new slot; the others through their empty-slot list
            dr = mode == 3 && S.reloc[tt];
            o = dr ? S.new_off[tt] : S.off[tt];
            a = S.hs[tt] + S.base[ 9 * tt + lane ];
            nn = S.new_np[tt];
        }
        s_off[tib][lane] = o;
        s_aux[tib][lane] = a;
        s_cap[tib][lane] = nn;
        s_dir[tib][lane] = dr;
        s_rank[tib][lane] = 0;
    }
    if ( WPT > 1 ) __syncthreads(); else __syncwarp();
    if ( active ) {
        const SpDev & S = *Sp;
        const RunDev & R = runs[ S.run ];
        const int t = it.tile, nxx = R.nxx, nxy = R.nxy;
        const int nl = S.nidx[t], off = S.off[t];
        // SU groups of 32 leavers in flight: their outbox loads, then their
        // slot lookups, then their stores
        for ( int k0 = sub * 32 * SU; k0 < nl; k0 += WPT * 32 * SU ) {
            uint32_t c[SU]; float xx[SU], xy[SU], ux[SU], uy[SU], uz[SU];
#pragma unroll
            for ( int u = 0; u < SU; u++ ) {
                const int k = k0 + u * 32 + lane;
                const size_t g = (size_t) off + k;
                c[u] = 0x80008000u;                   // (-32768, -32768): no leaver
                xx[u] = xy[u] = ux[u] = uy[u] = uz[u] = 0.f;
                if ( k < nl ) {
                    c[u] = S.B.cell[g]; xx[u] = S.B.xx[g]; xy[u] = S.B.xy[g];
                    ux[u] = S.B.ux[g]; uy[u] = S.B.uy[g]; uz[u] = S.B.uz[g];
                }
            }
            int slot[SU], dir[SU];
#pragma unroll
            for ( int u = 0; u < SU; u++ ) {
                const int k = k0 + u * 32 + lane;
                const int ix = cell_x( c[u] ), iy = cell_y( c[u] );
                const int xc = ( ix >= nxx ) - ( ix < 0 ), yc = ( iy >= nxy ) - ( iy < 0 );
                const int d = k < nl ? ( yc + 1 ) * 3 + xc + 1 : 9;
                const unsigned peers = __match_any_sync( 0xffffffffu, d );
                const int leader = __ffs( peers ) - 1;
                int b = 0;
                if ( d < 9 && lane == leader ) b = atomicAdd( &s_rank[tib][d], __popc( peers ) );
                b = __shfl_sync( peers, b, leader );
                dir[u] = d;
                slot[u] = -2;                          // -2: nothing to write
                if ( d < 9 && d != 4 && s_aux[tib][d] >= 0 ) {
                    // list entry and slot both below the target's new count
                    // (anything else means inconsistent counts: reported, the
                    // particle is not written)
                    const int r = s_aux[tib][d] + b + __popc( peers & lt );
                    slot[u] = r < s_cap[tib][d] ? ( s_dir[tib][d] ? r : S.aux[ (size_t) s_off[tib][d] + r ] ) : -1;
                }
            }
#pragma unroll
            for ( int u = 0; u < SU; u++ ) {
                if ( slot[u] == -2 ) continue;
                const int d = dir[u];
                if ( slot[u] >= 0 && slot[u] < s_cap[tib][d] ) {
                    const int ix = cell_x( c[u] ), iy = cell_y( c[u] );
                    const int xc = d % 3 - 1, yc = d / 3 - 1;
                    const size_t p = (size_t) s_off[tib][d] + slot[u];
                    S.A.cell[p] = pack_cell( ix - xc * nxx, iy - yc * nxy );
                    S.A.xx[p] = xx[u]; S.A.xy[p] = xy[u];
                    S.A.ux[p] = ux[u]; S.A.uy[p] = uy[u]; S.A.uz[p] = uz[u];
                } else {
                    atomicOr( R.status, ST_BAD_CELL );
                }
            }
        }
    }
    // every warp of the tile has read nidx before it is cleared
    if ( WPT > 1 ) __syncthreads(); else __syncwarp();
    if ( mode >= 0 && mode != 2 && sub == 0 && lane == 0 ) {
        const SpDev & S = *Sp;
        const int t = it.tile;
        S.np[t] = S.new_np[t];
        if ( mode == 1 || ( mode == 3 && S.reloc[t] ) ) { S.off[t] = S.new_off[t]; S.cap[t] = S.new_cap[t]; }
        S.nidx[t] = 0;
    }
    const int nr = rlist[0];
    for ( int k = 0; k < nr; k++ )
        if ( !( rlist[ 1 + k ] & RLIST_RELOCATE ) ) repack_in( sps[ rlist[ 1 + k ] ] );
}

// ---------------------------------------------------------------------------
// Injection (density.cpp): particles of a cell range appended to each tile.
// The order of the reference's sequential loops (i1, i0, cell) is kept with
// a block-wide ordered scan.
// ---------------------------------------------------------------------------

// Moving-window injection parameters that depend on the window's position
// (Injector rule: step position / slab limits / sphere centre relative to the
// window, density.cpp:418, 677-678, 937-941), computed on the device from a
// device copy of the window's move count so that a captured step replays
// with the right values; the count is advanced afterwards.  The arithmetic
// is the host's: motion = n_move * dx in double, rounded to float.
__global__ void k_inj_dyn( float * __restrict__ dyn, unsigned * __restrict__ n_move, int type,
                           float da, float db, float dx0, double mw_dx )
{
    const double motion = *n_move * mw_dx;
    const float refx = (float) motion;
    float a = 0.f, b = 0.f, cx = 0.f;
    if ( type == 2 ) a = ( da - refx ) / dx0;
    else if ( type == 3 ) { a = ( da - refx ) / dx0; b = ( db - refx ) / dx0; }
    else if ( type == 4 ) cx = da - refx;
    dyn[0] = a; dyn[1] = b; dyn[2] = cx;
    *n_move += 1;
}

__device__ __forceinline__ int inj_test( const InjRule & r, int shiftx, int shifty, int cx, int cy, float posx, float posy ) {
    float t;
    switch ( r.type ) {
    case 1: return 1;
    case 2:
        t = r.diry ? (float) ( ( shifty + cy ) + ( (double) posy + 0.5 ) ) : (float) ( ( shiftx + cx ) + ( (double) posx + 0.5 ) );
        return t > r.a;
    case 3:
        t = r.diry ? (float) ( ( shifty + cy ) + ( (double) posy + 0.5 ) ) : (float) ( ( shiftx + cx ) + ( (double) posx + 0.5 ) );
        return ( t >= r.a ) && ( t < r.b );
    case 4: {
        const float gx = (float) ( ( ( shiftx + cx ) + ( (double) posx + 0.5 ) ) * (double) r.dxx );
        const float gy = (float) ( ( ( shifty + cy ) + ( (double) posy + 0.5 ) ) * (double) r.dxy );
        return ( gx - r.cx ) * ( gx - r.cx ) + ( gy - r.cy ) * ( gy - r.cy ) < r.r2;
    }
    }
    return 0;
}

__device__ __forceinline__ bool inj_tile_range( const InjRule & r, int tx, int ty, int nxx, int nxy,
                                                int & ri0, int & ri1, int & rj0, int & rj1 ) {
    ri0 = r.range[0] - tx * nxx; ri1 = r.range[1] - tx * nxx;
    rj0 = r.range[2] - ty * nxy; rj1 = r.range[3] - ty * nxy;
    if ( ( ri0 < nxx ) && ( ri1 >= 0 ) && ( rj0 < nxy ) && ( rj1 >= 0 ) ) {
        if ( ri0 < 0 ) ri0 = 0;
        if ( rj0 < 0 ) rj0 = 0;
        if ( ri1 >= nxx ) ri1 = nxx - 1;
        if ( rj1 >= nxy ) rj1 = nxy - 1;
        return true;
    }
    return false;
}

constexpr int INJ_THREADS = 256;

// count == 1: write the number of particles to inject per tile to S.extra
// count == 0: inject them after the existing particles of each tile
__global__ void __launch_bounds__( INJ_THREADS )
k_inject( int sp, const SpDev * __restrict__ sps, const RunDev * __restrict__ runs, InjRule r, int count,
          int tx0, int ntx_r, int ty0 )
{
    const SpDev & S = sps[sp];
    const RunDev & R = runs[ S.run ];
    // CTA b covers tile (tx0 + b % ntx_r, ty0 + b / ntx_r) of the range's tiles
    const int t = ( ty0 + (int) blockIdx.x / ntx_r ) * R.ntx + tx0 + (int) blockIdx.x % ntx_r;
    const int tx = t % R.ntx, ty = t / R.ntx;
    const int nxx = R.nxx, nxy = R.nxy;
    if ( r.dyn ) { r.a = r.dyn[0]; r.b = r.dyn[1]; r.cx = r.dyn[2]; }
    int ri0, ri1, rj0, rj1;
    const bool in_range = ( tx < r.tx_limit ) && inj_tile_range( r, tx, ty, nxx, nxy, ri0, ri1, rj0, rj1 );
    if ( !in_range ) {
        if ( count && threadIdx.x == 0 ) S.extra[t] = 0;
        return;
    }
    const int row = ri1 - ri0 + 1, vol = ( rj1 - rj0 + 1 ) * row;
    const int total = vol * r.ppcx * r.ppcy;
    const int shiftx = tx * nxx, shifty = ty * nxy;
    const double dpcx = 1.0 / r.ppcx, dpcy = 1.0 / r.ppcy;
    __shared__ long long s_tot;
    int run = 0;
    const int base = count ? 0 : S.np[t];
    const int off = S.off[t];
    for ( int L0 = 0; L0 < total; L0 += INJ_THREADS ) {
        const int L = L0 + threadIdx.x;
        int inj = 0, cx = 0, cy = 0; float posx = 0, posy = 0;
        if ( L < total ) {
            const int idx = L % vol, pidx = L / vol;
            const int i0 = pidx % r.ppcx, i1 = pidx / r.ppcx;
            posx = (float) ( dpcx * ( i0 + 0.5 ) - 0.5 );
            posy = (float) ( dpcy * ( i1 + 0.5 ) - 0.5 );
            cx = idx % row + ri0; cy = idx / row + rj0;
            inj = inj_test( r, shiftx, shifty, cx, cy, posx, posy );
        }
        long long pre = block_exscan< INJ_THREADS >( inj, &s_tot );
        __syncthreads();
        const int tot = (int) s_tot;
        if ( !count && inj ) {
            const size_t g = (size_t) off + base + run + pre;
            S.A.cell[g] = pack_cell( cx, cy );
            S.A.xx[g] = posx; S.A.xy[g] = posy;
            S.A.ux[g] = 0.f; S.A.uy[g] = 0.f; S.A.uz[g] = 0.f;
        }
        run += tot;
        __syncthreads();
    }
    if ( threadIdx.x == 0 ) {
        if ( count ) S.extra[t] = run;
        else S.np[t] = base + run;
    }
}

// ---------------------------------------------------------------------------
// Conversion between the slot layout and the reference's packed layout
// (ix int2, x float2, u float3; tiles contiguous at packed offsets).
// ---------------------------------------------------------------------------
__global__ void k_pack( int sp, const SpDev * __restrict__ sps, const int * __restrict__ poff,
                        int2 * __restrict__ ix, float2 * __restrict__ x, float * __restrict__ u )
{
    const SpDev & S = sps[sp];
    const int t = blockIdx.x;
    const int np = S.np[t], off = S.off[t], po = poff[t];
    for ( int i = threadIdx.x; i < np; i += blockDim.x ) {
        const size_t g = (size_t) off + i, d = (size_t) po + i;
        const uint32_t c = S.A.cell[g];
        ix[d] = make_int2( cell_x( c ), cell_y( c ) );
        x[d] = make_float2( S.A.xx[g], S.A.xy[g] );
        u[3*d] = S.A.ux[g]; u[3*d+1] = S.A.uy[g]; u[3*d+2] = S.A.uz[g];
    }
}

__global__ void k_unpack( int sp, const SpDev * __restrict__ sps, const int * __restrict__ poff, int t0, long long pbase,
                          const int2 * __restrict__ ix, const float2 * __restrict__ x, const float * __restrict__ u )
{
    const SpDev & S = sps[sp];
    const int t = t0 + blockIdx.x;
    const int np = S.np[t], off = S.off[t];
    const long long po = poff[t] - pbase;
    for ( int i = threadIdx.x; i < np; i += blockDim.x ) {
        const size_t g = (size_t) off + i, s = (size_t) po + i;
        S.A.cell[g] = pack_cell( ix[s].x, ix[s].y );
        S.A.xx[g] = x[s].x; S.A.xy[g] = x[s].y;
        S.A.ux[g] = u[3*s]; S.A.uy[g] = u[3*s+1]; S.A.uz[g] = u[3*s+2];
    }
}

// Species::gather (particles.cpp:16-200): value per particle at packed offsets,
// optionally scaled as fma(scale.x, val, scale.y).
__global__ void k_gather( int sp, const SpDev * __restrict__ sps, const RunDev * __restrict__ runs,
                          const int * __restrict__ poff, int quant, float sx, float sy, int scaled,
                          float * __restrict__ out )
{
    const SpDev & S = sps[sp];
    const RunDev & R = runs[ S.run ];
    const int t = blockIdx.x;
    const int tx = t % R.ntx, ty = t / R.ntx;
    const int np = S.np[t], off = S.off[t], po = poff[t];
    for ( int i = threadIdx.x; i < np; i += blockDim.x ) {
        const size_t g = (size_t) off + i;
        float val;
        switch ( quant ) {
        case 0: val = ( tx * R.nxx + cell_x( S.A.cell[g] ) ) + ( 0.5f + S.A.xx[g] ); break;
        case 1: val = ( ty * R.nxy + cell_y( S.A.cell[g] ) ) + ( 0.5f + S.A.xy[g] ); break;
        case 2: val = S.A.ux[g]; break;
        case 3: val = S.A.uy[g]; break;
        default: val = S.A.uz[g]; break;
        }
        out[ (size_t) po + i ] = scaled ? __fmaf_rn( sx, val, sy ) : val;
    }
}

// Charge deposit (species.cpp:2348-2399) into a tiled scalar grid with guard
// cells {0,1}; per-tile shared-memory accumulation, then a store of the tile.
__global__ void k_dep_charge( int sp, const SpDev * __restrict__ sps, const RunDev * __restrict__ runs,
                              float * __restrict__ charge, int cextx, int cvol )
{
    extern __shared__ float sc[];
    const SpDev & S = sps[sp];
    const int t = blockIdx.x;
    for ( int i = threadIdx.x; i < cvol; i += blockDim.x ) sc[i] = 0.f;
    __syncthreads();
    const int np = S.np[t], off = S.off[t];
    const float q = S.q;
    for ( int i = threadIdx.x; i < np; i += blockDim.x ) {
        const size_t g = (size_t) off + i;
        const uint32_t c = S.A.cell[g];
        const int idx = cell_y( c ) * cextx + cell_x( c );
        const float xx = S.A.xx[g], xy = S.A.xy[g];
        const float s0x = 0.5f - xx, s1x = 0.5f + xx, s0y = 0.5f - xy, s1y = 0.5f + xy;
        atomicAdd( sc + idx, s0y * s0x * q );
        atomicAdd( sc + idx + 1, s0y * s1x * q );
        atomicAdd( sc + idx + cextx, s1y * s0x * q );
        atomicAdd( sc + idx + 1 + cextx, s1y * s1x * q );
    }
    __syncthreads();
    for ( int i = threadIdx.x; i < cvol; i += blockDim.x ) charge[ (size_t) t * cvol + i ] += sc[i];
    (void) runs;
}

// Phase-space density of one species (dep_pha1_kernel species.cpp:2579-2620,
// dep_pha2_kernel 2786-2852): every particle adds linear weights to two (1D)
// or four (2D) bins; bins k with k < 0 or k >= size-1 receive nothing (the
// reference's bound, which leaves the last bin empty).  Quantities:
// 0 x, 1 y (cell units, tile shift included), 2 ux, 3 uy, 4 uz.  With
// PhaSpec::smem the CTA accumulates into a shared-memory copy of the whole
// phase space and adds its non-zero bins to the output at the end.
__device__ __forceinline__ float pha_quant( int q, int shiftx, int shifty, uint32_t c,
                                            float xx, float xy, float ux, float uy, float uz ) {
    switch ( q ) {
    case 0:  return (float) ( shiftx + cell_x( c ) ) + ( xx + 0.5f );
    case 1:  return (float) ( shifty + cell_y( c ) ) + ( xy + 0.5f );
    case 2:  return ux;
    case 3:  return uy;
    default: return uz;
    }
}

__global__ void k_phasespace( int sp, const SpDev * __restrict__ sps, const RunDev * __restrict__ runs,
                              PhaSpec p, float * __restrict__ out )
{
    extern __shared__ float sh[];
    const SpDev & S = sps[sp];
    const RunDev & R = runs[ S.run ];
    const bool two = p.q1 >= 0;
    const int nbins = p.n0 * ( two ? p.n1 : 1 );
    float * h = p.smem ? sh : out;
    if ( p.smem ) {
        for ( int i = threadIdx.x; i < nbins; i += blockDim.x ) sh[i] = 0.f;
        __syncthreads();
    }
    const int ntiles = R.ntx * R.nty;
    for ( int t = blockIdx.x; t < ntiles; t += gridDim.x ) {
        const int np = S.np[t], off = S.off[t];
        const int shiftx = ( t % R.ntx ) * R.nxx, shifty = ( t / R.ntx ) * R.nxy;
        for ( int i = threadIdx.x; i < np; i += blockDim.x ) {
            const size_t g = (size_t) off + i;
            const uint32_t c = S.A.cell[g];
            const float xx = S.A.xx[g], xy = S.A.xy[g], ux = S.A.ux[g], uy = S.A.uy[g], uz = S.A.uz[g];
            const float n0 = ( pha_quant( p.q0, shiftx, shifty, c, xx, xy, ux, uy, uz ) - p.r0 ) * p.rdx0 - 0.5f;
            const int k0 = int( n0 + 1 ) - 1;
            const float w0 = n0 - k0;
            const bool a0 = k0 >= 0 && k0 < p.n0 - 1, b0 = k0 + 1 >= 0 && k0 + 1 < p.n0 - 1;
            if ( !two ) {
                if ( a0 ) atomicAdd( h + k0, ( 1 - w0 ) * p.norm );
                if ( b0 ) atomicAdd( h + k0 + 1, w0 * p.norm );
            } else {
                const float n1 = ( pha_quant( p.q1, shiftx, shifty, c, xx, xy, ux, uy, uz ) - p.r1 ) * p.rdx1 - 0.5f;
                const int k1 = int( n1 + 1 ) - 1;
                const float w1 = n1 - k1;
                const bool a1 = k1 >= 0 && k1 < p.n1 - 1, b1 = k1 + 1 >= 0 && k1 + 1 < p.n1 - 1;
                if ( a0 && a1 ) atomicAdd( h + k1 * p.n0 + k0,           ( 1 - w0 ) * ( 1 - w1 ) * p.norm );
                if ( b0 && a1 ) atomicAdd( h + k1 * p.n0 + k0 + 1,       w0 * ( 1 - w1 ) * p.norm );
                if ( a0 && b1 ) atomicAdd( h + ( k1 + 1 ) * p.n0 + k0,   ( 1 - w0 ) * w1 * p.norm );
                if ( b0 && b1 ) atomicAdd( h + ( k1 + 1 ) * p.n0 + k0 + 1, w0 * w1 * p.norm );
            }
        }
    }
    if ( p.smem ) {
        __syncthreads();
        for ( int i = threadIdx.x; i < nbins; i += blockDim.x )
            if ( sh[i] != 0.f ) atomicAdd( out + i, sh[i] );
    }
}

// Per-item energy sums reduced per species in item order (deterministic).
__global__ void k_energy_sum( const SpDev * __restrict__ sps, int sp, int nitems, double * __restrict__ out )
{
    const SpDev & S = sps[sp];
    __shared__ double s[256];
    double a = 0.0;
    const int per = ( nitems + blockDim.x - 1 ) / blockDim.x;
    const int i0 = threadIdx.x * per, i1 = min( nitems, i0 + per );
    for ( int i = i0; i < i1; i++ ) a += S.energy[i];
    s[ threadIdx.x ] = a;
    __syncthreads();
    if ( threadIdx.x == 0 ) {
        double tot = 0.0;
        for ( int i = 0; i < (int) blockDim.x; i++ ) tot += s[i];
        *out = tot;
    }
}

// Tile counts: np_total and np_max_tile
__global__ void k_np_stats( const SpDev * __restrict__ sps, int sp, unsigned long long * __restrict__ out )
{
    const SpDev & S = sps[sp];
    __shared__ unsigned long long s_sum[256];
    __shared__ unsigned s_max[256];
    unsigned long long a = 0; unsigned m = 0;
    for ( int t = threadIdx.x; t < S.ntiles; t += blockDim.x ) { a += S.np[t]; m = max( m, (unsigned) S.np[t] ); }
    s_sum[ threadIdx.x ] = a; s_max[ threadIdx.x ] = m;
    __syncthreads();
    if ( threadIdx.x == 0 ) {
        unsigned long long tot = 0; unsigned mx = 0;
        for ( int i = 0; i < (int) blockDim.x; i++ ) { tot += s_sum[i]; mx = max( mx, s_max[i] ); }
        out[0] = tot; out[1] = mx;
    }
}

// ---------------------------------------------------------------------------
// In-tile reorder (option "reorder": every n steps)
// ---------------------------------------------------------------------------
// Particles keep their slot while they move between the cells of their tile,
// so after some tens of steps the 32 lanes of a warp of the particle kernel
// hold particles in random cells of the tile, and its shared-memory field
// gathers and tile-current atomics meet about 3.5-way bank conflicts instead of
// the 2-way of the injection order.  This kernel puts each tile back into
// cell round-robin order: particles sorted by (rank within their cell, cell),
// so round r lists one particle of every cell that holds more than r, in
// ascending cell order, and consecutive lanes again see consecutive cells.
// The rank comes from a shared-memory counter per cell (its order between
// particles of one cell is arbitrary) and is kept beside the cell index in
// the shared copy of the tile's cells, which are read once; the position of
// (r, c) is the number of particles in the rounds before r plus the cells
// before c in round r, counted with a bit mask of the cells present in each
// round.  The tile is then permuted in place one particle array at a time
// through shared memory (coalesced loads and stores, 8 bytes of traffic per
// particle and array; the cell words are rebuilt from the cell indices).
// One CTA per tile, either 1024 threads alone on an SM or, for tiles that
// fit half of the shared memory, 512 threads with two CTAs per SM (one
// CTA's loads and stores overlap the other's counting).  Tiles with more
// particles than fit, with more particles in one cell than there are rounds,
// or with a particle outside the tile are left as they are.
template < int NT >
__global__ void __launch_bounds__( NT, 1024 / NT )
k_reorder( const Item * __restrict__ items, const SpDev * __restrict__ sps, const RunDev * __restrict__ runs,
           int max_rounds, int np_min, int np_max )
{
    extern __shared__ __align__( 16 ) unsigned char smem_raw[];
    const Item it = items[ blockIdx.x ];
    const SpDev & S = sps[ it.sp ];
    const RunDev & R = runs[ S.run ];
    const int t = it.tile;
    const int np = S.np[t];
    if ( np < np_min || np > np_max ) return;
    const size_t off = S.off[t];
    const int nxx = R.nxx, nxy = R.nxy, ncell = nxx * nxy;
    const int ncw = ( ncell + 31 ) >> 5;
    // shared memory: [buf: np_max words][inv: np_max 16-bit][cnt: ncw*32]
    //                [base: max_rounds+1][flags: 4][masks: max_rounds*ncw words][word prefix: max_rounds*ncw 16-bit]
    uint32_t * buf = reinterpret_cast<uint32_t *>( smem_raw );
    uint16_t * inv = reinterpret_cast<uint16_t *>( buf + np_max );
    int * cnt = reinterpret_cast<int *>( inv + np_max );
    int * base = cnt + ncw * 32;
    int * flags = base + max_rounds + 1;
    uint32_t * masks = reinterpret_cast<uint32_t *>( flags + 4 );
    uint16_t * wpre = reinterpret_cast<uint16_t *>( masks + max_rounds * ncw );
    const int n4 = np >> 2;

    // the tile's cells, read once into shared memory
    {
        const uint32_t * g = S.A.cell + off;
#pragma unroll 4
        for ( int v = threadIdx.x; v < n4; v += NT )
            reinterpret_cast<uint4 *>( buf )[v] = reinterpret_cast<const uint4 *>( g )[v];
        for ( int p = 4 * n4 + threadIdx.x; p < np; p += NT ) buf[p] = g[p];
    }
    for ( int c = threadIdx.x; c < ncw * 32; c += NT ) cnt[c] = 0;
    if ( threadIdx.x == 0 ) { flags[0] = 0; flags[1] = 0; }
    __syncthreads();
    // rank within the cell, kept as (cell index | rank << 16)
    for ( int i = threadIdx.x; i < np; i += NT ) {
        const uint32_t cl = buf[i];
        const int ix = cell_x( cl ), iy = cell_y( cl );
        if ( ix < 0 || ix >= nxx || iy < 0 || iy >= nxy ) { flags[0] = 1; continue; }
        const int c = ix + nxx * iy;
        const int r = atomicAdd( cnt + c, 1 );
        if ( r >= max_rounds ) flags[0] = 1;
        else { atomicMax( flags + 1, r + 1 ); buf[i] = (uint32_t) c | ( (uint32_t) r << 16 ); }
    }
    __syncthreads();
    if ( flags[0] ) return;
    const int nround = flags[1];
    // cells present in each round, one 32-cell word per warp pass
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = NT / 32;
    for ( int w = warp; w < ncw; w += NW ) {
        const int n = cnt[ w * 32 + lane ];
        for ( int r = 0; r < nround; r++ ) {
            const uint32_t m = __ballot_sync( 0xffffffffu, n > r );
            if ( lane == 0 ) masks[ r * ncw + w ] = m;
        }
    }
    __syncthreads();
    // per round: prefix of the word populations, and the round's size
    for ( int r = threadIdx.x; r < nround; r += NT ) {
        int a = 0;
        for ( int w = 0; w < ncw; w++ ) { wpre[ r * ncw + w ] = (uint16_t) a; a += __popc( masks[ r * ncw + w ] ); }
        base[r] = a;
    }
    __syncthreads();
    if ( warp == 0 ) {
        // exclusive scan of the round sizes, 32 rounds per pass
        int carry = 0;
        for ( int r0 = 0; r0 < nround; r0 += 32 ) {
            const int r = r0 + lane;
            const int v = r < nround ? base[r] : 0;
            int incl = v;
#pragma unroll
            for ( int o = 1; o < 32; o <<= 1 ) {
                const int y = __shfl_up_sync( 0xffffffffu, incl, o );
                if ( lane >= o ) incl += y;
            }
            if ( r < nround ) base[r] = carry + incl - v;
            carry += __shfl_sync( 0xffffffffu, incl, 31 );
        }
    }
    __syncthreads();
    for ( int i = threadIdx.x; i < np; i += NT ) {
        const uint32_t e = buf[i];
        const int c = e & 0xffff, r = e >> 16;
        const int w = c >> 5;
        const int pos = base[r] + wpre[ r * ncw + w ] + __popc( masks[ r * ncw + w ] & ( ( 1u << ( c & 31 ) ) - 1u ) );
        inv[pos] = (uint16_t) i;
    }
    __syncthreads();
    // the cells, rebuilt from the cell indices
    {
        uint32_t * g = S.A.cell + off;
#pragma unroll 4
        for ( int v = threadIdx.x; v < n4; v += NT ) {
            uint32_t q[4];
#pragma unroll
            for ( int u = 0; u < 4; u++ ) {
                const int c = buf[ inv[ 4 * v + u ] ] & 0xffff;
                q[u] = pack_cell( c % nxx, c / nxx );
            }
            reinterpret_cast<uint4 *>( g )[v] = make_uint4( q[0], q[1], q[2], q[3] );
        }
        for ( int p = 4 * n4 + threadIdx.x; p < np; p += NT ) {
            const int c = buf[ inv[p] ] & 0xffff;
            g[p] = pack_cell( c % nxx, c / nxx );
        }
    }
    // then each other particle array in place through shared memory
    uint32_t * arr[5] = { reinterpret_cast<uint32_t *>( S.A.xx ), reinterpret_cast<uint32_t *>( S.A.xy ),
                          reinterpret_cast<uint32_t *>( S.A.ux ), reinterpret_cast<uint32_t *>( S.A.uy ),
                          reinterpret_cast<uint32_t *>( S.A.uz ) };
    for ( int a = 0; a < 5; a++ ) {
        uint32_t * g = arr[a] + off;
        __syncthreads();
#pragma unroll 4
        for ( int v = threadIdx.x; v < n4; v += NT )
            reinterpret_cast<uint4 *>( buf )[v] = reinterpret_cast<const uint4 *>( g )[v];
        for ( int p = 4 * n4 + threadIdx.x; p < np; p += NT ) buf[p] = g[p];
        __syncthreads();
#pragma unroll 4
        for ( int v = threadIdx.x; v < n4; v += NT ) {
            const int p = 4 * v;
            reinterpret_cast<uint4 *>( g )[v] = make_uint4( buf[ inv[p] ], buf[ inv[p + 1] ], buf[ inv[p + 2] ], buf[ inv[p + 3] ] );
        }
        for ( int p = 4 * n4 + threadIdx.x; p < np; p += NT ) g[p] = buf[ inv[p] ];
    }
}

}  // namespace zb

// ---------------------------------------------------------------------------
// Launch wrappers (host side of this translation unit)
// ---------------------------------------------------------------------------
namespace zb {

size_t particle_smem_bytes( int tile_vol, int jacc ) {
    return (size_t) ( jacc ? 12 : 9 ) * tile_vol * sizeof( float ) + 8 + ( PK_THREADS / 32 ) * sizeof( double ) +
           ( PK_THREADS / 32 ) * sizeof( CrossQueue );
}

typedef void ( *pk_fn )( const Item *, const SpDev *, const RunDev *, const int * );

static pk_fn pick_particle_kernel( int push, int move, int detect, int jacc, int tile_n ) {
    if ( tile_n == 16 && move == 2 && detect && ( push == 1 || push == 2 ) ) {
        if ( jacc == 0 ) return push == 1 ? k_particles< 1, 2, true, float, 16 > : k_particles< 2, 2, true, float, 16 >;
        if ( jacc == 1 ) return push == 1 ? k_particles< 1, 2, true, double, 16 > : k_particles< 2, 2, true, double, 16 >;
        return push == 1 ? k_particles< 1, 2, true, int, 16 >
                         : k_particles< 2, 2, true, int, 16 >;
    }
    if ( jacc == 1 && move == 2 ) {
#define PKD( P, M, D ) if ( push == P && move == M && detect == D ) return k_particles< P, M, D, double >;
        PKD( 1, 2, true ) PKD( 2, 2, true ) PKD( 0, 2, true )
#undef PKD
        return nullptr;
    }
    if ( jacc == 2 && move == 2 ) {
#define PKX( P, M, D ) if ( push == P && move == M && detect == D ) return k_particles< P, M, D, int >;
        PKX( 1, 2, true ) PKX( 2, 2, true ) PKX( 0, 2, true )
#undef PKX
        return nullptr;
    }
#define PK( P, M, D ) if ( push == P && move == M && detect == D ) return k_particles< P, M, D >;
    PK( 1, 2, true ) PK( 2, 2, true )
    PK( 1, 0, false ) PK( 2, 0, false )
    PK( 0, 2, true ) PK( 0, 1, true ) PK( 0, 0, true )
    PK( 1, 1, true ) PK( 2, 1, true )
#undef PK
    return nullptr;
}

cudaError_t launch_particles( cudaStream_t st, int push, int move, int detect, const Item * items, int nitems,
                              const SpDev * sps, const RunDev * runs, const int * shifts, int max_tile_vol,
                              int jacc, int tile_n ) {
    if ( move != 2 ) jacc = 0;
    pk_fn f = pick_particle_kernel( push, move, detect, jacc, tile_n );
    if ( !f ) return cudaErrorInvalidValue;
    const size_t smem = particle_smem_bytes( max_tile_vol, jacc );
    if ( smem > 48 * 1024 )
        cudaFuncSetAttribute( (const void *) f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem );
    if ( nitems <= 0 ) return cudaSuccess;
    f<<< nitems, PK_THREADS, smem, st >>>( items, sps, runs, shifts );
    return cudaGetLastError();
}

cudaError_t launch_sort( cudaStream_t st, const Item * items, int nitems, const SpDev * sps,
                         const int * species_list, int nspecies, const RunDev * runs, int use_extra, int * rlist ) {
    if ( nitems <= 0 ) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice( &dev );
    cudaDeviceGetAttribute( &sms, cudaDevAttrMultiProcessorCount, dev );
    k_sort_check<<< ( nitems + CHECK_THREADS - 1 ) / CHECK_THREADS, CHECK_THREADS, 0, st >>>( items, nitems, sps, runs,
                                                                                         use_extra, rlist );
    k_sort_plan<<< nspecies, PLAN_THREADS, 0, st >>>( sps, species_list, runs, use_extra, rlist );
    // a warp per tile, unless the tiles are too few to occupy the GPU's SMs
    // (then they are large, and get a CTA each); the grid covers the GPU at
    // least once for the repack's grid-stride loops
    const bool wide = nitems < sms * 16;
    const int tpb = wide ? 1 : SORT_WARPS;
    const int nb = std::max( ( nitems + tpb - 1 ) / tpb, 4 * sms );
    if ( wide ) {
        k_sort_local< SORT_WARPS ><<< nb, SORT_THREADS, 0, st >>>( items, nitems, sps, rlist, runs );
        k_sort_scatter< SORT_WARPS ><<< nb, SORT_THREADS, 0, st >>>( items, nitems, sps, rlist, runs );
    } else {
        k_sort_local< 1 ><<< nb, SORT_THREADS, 0, st >>>( items, nitems, sps, rlist, runs );
        k_sort_scatter< 1 ><<< nb, SORT_THREADS, 0, st >>>( items, nitems, sps, rlist, runs );
    }
    return cudaGetLastError();
}

cudaError_t launch_inj_dyn( cudaStream_t st, float * dyn, unsigned * n_move, int type, float da, float db,
                            float dx0, double mw_dx ) {
    k_inj_dyn<<< 1, 1, 0, st >>>( dyn, n_move, type, da, db, dx0, mw_dx );
    return cudaGetLastError();
}

// Tiles [tx0, tx1] x [ty0, ty1] hold the injection range; the caller clears
// the other tiles' counts (count mode).
cudaError_t launch_inject( cudaStream_t st, int sp, int tx0, int tx1, int ty0, int ty1, const SpDev * sps,
                           const RunDev * runs, const InjRule & r, int count ) {
    const int nx = tx1 - tx0 + 1, ny = ty1 - ty0 + 1;
    if ( nx <= 0 || ny <= 0 ) return cudaSuccess;
    k_inject<<< nx * ny, INJ_THREADS, 0, st >>>( sp, sps, runs, r, count, tx0, nx, ty0 );
    return cudaGetLastError();
}

cudaError_t launch_pack( cudaStream_t st, int sp, int ntiles, const SpDev * sps, const int * poff,
                         int2 * ix, float2 * x, float * u ) {
    k_pack<<< ntiles, 256, 0, st >>>( sp, sps, poff, ix, x, u );
    return cudaGetLastError();
}

// Tiles [t0, t0 + ntiles) from packed arrays holding the particles from
// packed offset pbase on.
cudaError_t launch_unpack( cudaStream_t st, int sp, int t0, int ntiles, const SpDev * sps, const int * poff,
                           long long pbase, const int2 * ix, const float2 * x, const float * u ) {
    if ( ntiles <= 0 ) return cudaSuccess;
    k_unpack<<< ntiles, 256, 0, st >>>( sp, sps, poff, t0, pbase, ix, x, u );
    return cudaGetLastError();
}

cudaError_t launch_gather( cudaStream_t st, int sp, int ntiles, const SpDev * sps, const RunDev * runs,
                           const int * poff, int quant, float sx, float sy, int scaled, float * out ) {
    k_gather<<< ntiles, 256, 0, st >>>( sp, sps, runs, poff, quant, sx, sy, scaled, out );
    return cudaGetLastError();
}

cudaError_t launch_dep_charge( cudaStream_t st, int sp, int ntiles, const SpDev * sps, const RunDev * runs,
                               float * charge, int cextx, int cvol ) {
    k_dep_charge<<< ntiles, 256, cvol * sizeof( float ), st >>>( sp, sps, runs, charge, cextx, cvol );
    return cudaGetLastError();
}

cudaError_t launch_phasespace( cudaStream_t st, int sp, int ntiles, const SpDev * sps, const RunDev * runs,
                              PhaSpec p, float * out ) {
    const int nbins = p.n0 * ( p.q1 >= 0 ? p.n1 : 1 );
    const size_t smem = (size_t) nbins * sizeof( float );
    // a private copy per CTA when the phase space fits in shared memory
    p.smem = smem <= 200 * 1024;
    if ( p.smem && smem > 48 * 1024 )
        cudaFuncSetAttribute( (const void *) k_phasespace, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem );
    const int grid = p.smem ? std::min( ntiles, 2 * 148 ) : ntiles;
    k_phasespace<<< grid, 256, p.smem ? smem : 0, st >>>( sp, sps, runs, p, out );
    return cudaGetLastError();
}

cudaError_t launch_energy_sum( cudaStream_t st, const SpDev * sps, int sp, int nitems, double * out ) {
    k_energy_sum<<< 1, 256, 0, st >>>( sps, sp, nitems, out );
    return cudaGetLastError();
}

// Rounds (the most particles in one cell) and particles per tile that
// k_reorder handles for tiles of up to max_cells cells: 1024 threads in
// 227 KB of shared memory, or two CTAs of 512 threads per SM in 113 KB each
// (tiles of up to 256 cells with fewer particles than fit there; the large
// configuration takes the larger tiles in a second launch).
cudaError_t launch_reorder( cudaStream_t st, const Item * items, int nitems, const SpDev * sps, const RunDev * runs,
                            int max_cells ) {
    if ( nitems <= 0 ) return cudaSuccess;
    const int ncw = ( max_cells + 31 ) / 32;
    auto fixed_bytes = [&]( int rounds ) {
        return (size_t) ncw * 32 * 4 + ( rounds + 1 ) * 4 + 16 + (size_t) rounds * ncw * 6;
    };
    // per particle: one 4-byte word (the cells with their ranks, then the
    // array being permuted) and a 16-bit source index
    auto np_fit = [&]( size_t budget, int rounds ) -> int {
        const size_t fx = fixed_bytes( rounds );
        if ( fx + 64 * 6 > budget ) return 0;
        return (int) std::min<size_t>( 65532, ( ( budget - fx ) / 6 ) & ~(size_t) 7 );
    };
    int np_lo = 64;
    if ( max_cells <= 256 ) {
        const int rounds = 127;
        const int np2 = np_fit( 113 * 1024, rounds );
        if ( np2 >= 1024 ) {
            const size_t smem = (size_t) np2 * 6 + fixed_bytes( rounds );
            cudaFuncSetAttribute( (const void *) k_reorder<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem );
            k_reorder<512><<< nitems, 512, smem, st >>>( items, sps, runs, rounds, np_lo, np2 );
            const cudaError_t e = cudaGetLastError();
            if ( e != cudaSuccess ) return e;
            np_lo = np2 + 1;
        }
    }
    const int rounds = std::max( 1, std::min( 511, ( 32 * 1024 ) / ( 6 * ncw ) - 1 ) );
    const int np1 = np_fit( 227 * 1024, rounds );
    if ( np1 < np_lo ) return cudaSuccess;
    const size_t smem = (size_t) np1 * 6 + fixed_bytes( rounds );
    cudaFuncSetAttribute( (const void *) k_reorder<1024>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem );
    k_reorder<1024><<< nitems, 1024, smem, st >>>( items, sps, runs, rounds, np_lo, np1 );
    return cudaGetLastError();
}

cudaError_t launch_np_stats( cudaStream_t st, const SpDev * sps, int sp, unsigned long long * out ) {
    k_np_stats<<< 1, 256, 0, st >>>( sps, sp, out );
    return cudaGetLastError();
}

}  // namespace zb
