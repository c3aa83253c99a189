// zpic_dev.cuh -- device-side descriptors and helpers shared by the em2d kernels.
//
// Data layout in HBM
//   fields  : per-tile float3 blocks with guard cells {1,2} on both axes, the
//             reference's tiled layout (grid.h:77-92): tile_vol =
//             roundup4(ext_x*ext_y) cells per tile, cell (0,0) at gc_off.
//   particles: six SoA arrays per species, one slot per tile
//             [off[t], off[t]+cap[t]) with np[t] used entries; off[] and cap[]
//             are multiples of 4 so a thread loads 4 particles with 128-bit
//             accesses.  cell = (int16 ix.x) | (int16 ix.y) << 16.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace zb {

// Status bits written by kernels (host reads them after synchronising).
enum : int {
    ST_WAIT_TIMEOUT   = 1,    // a bounded mbarrier / bulk-copy wait gave up
    ST_STAGE_OVERFLOW = 2,    // sort staging buffer too small (repack taken)
    ST_CAPACITY       = 4,    // particle buffer too small for the new layout
    ST_BAD_CELL       = 8,    // a particle moved more than one tile (invalid input)
};

// Per-simulation (run) geometry and field buffers.
struct RunDev {
    int ntx, nty, nxx, nxy;       // tiles, tile size
    int extx, exty;               // tile size with guard cells
    int gc_off;                   // offset of cell (0,0) inside a tile block
    int tile_vol;                 // cells per tile block
    float * E; float * B;         // float3 per cell
    float * J;                    // final current (after guard-cell exchange)
    float * Jdep;                 // raw deposits (tile-local sums incl. guard cells)
    float * bcol;                 // B of every tile's first interior column (ntiles x nxy float3),
                                  // saved by the Yee kernel ahead of a window shift
    int emf_perx, emf_pery;       // E/B periodic flags (grid::periodic)
    int cur_perx, cur_pery;       // J periodic flags
    float dtx, dty, dtx2, dty2;   // Yee coefficients dt/dx, dt/dy and halves (emf.cpp:524-525)
    float dt;                     // dt as passed to yeeJ_e (FP32)
    int emf_bc[4];                // emf::bc
    int cur_bc[4];                // current::bc
    int * status;                 // ST_* bits
    int wait_limit;               // polls of a bounded wait before it gives up (option "wait_limit")
};

// Particle arrays of one buffer (A, repack buffer B or staging).
struct PartArrays {
    uint32_t * cell;
    float * xx; float * xy;
    float * ux; float * uy; float * uz;
};

// Per-species state.
struct SpDev {
    int run;
    int ntiles;
    int nchunk;                   // CTAs per tile in the particle kernel (at most)
    int chunk_target;             // particles per CTA: a tile uses ceil(np / target) of its
                                  // nchunk CTAs (0: all of them)
    int max_part;                 // capacity of A and B
    PartArrays A, B;              // particles (tile slots) and second buffer (leaver outbox, repack target)
    int * np; int * off; int * cap;          // tile slots of A
    int * nidx;                   // [ntiles] leavers per tile
    int * idx;                    // [max_part] local index of leavers, at off[t]+k
    int * aux; int * aux2;        // [max_part] empty-slot / stayer lists, at off[t]+k
    int * cnt;                    // [9 ntiles] leavers per tile and direction (particle kernel)
    int * base;                   // [9 ntiles] first incoming rank per direction (sort check)
    int * in_cnt;                 // [ntiles] incoming particles (sort check)
    int * hs;                     // [ntiles] stayers moved down inside the tile (sort); in a repack:
                                  // packed position of each tile's first particle, old layout
    int * overflow;               // [1] a tile's new count exceeds its slot (sort check)
    int * reloc;                  // [ntiles] 1: the tile outgrew its slot and moves to the pool (sort check)
    int * pool;                   // [1] start of the free pool after the last slot (pool ends at max_part)
    int * rel_tile;               // [ntiles] relocated tiles of the current sort, in tile order (plan)
    int * rel_start;              // [ntiles + 1] their particles' packed starts; [nrel] = total (plan)
    int * rel_n;                  // [1] number of relocated tiles (plan)
    int * stage_cnt;              // [ntiles] repack fill counters
    int * new_off; int * new_cap; int * new_np;  // [ntiles] new counts, repack layout
    int * extra;                  // [ntiles] room to reserve for injection (or nullptr)
    int * mode;                   // [1] 0 in-place sort, 1 repack, 2 no room, 3 in place with relocated tiles
    double * energy;              // [ntiles*nchunk] per work-item kinetic energy sums
    unsigned long long * nmove;   // [0] pushes counter, [1] repacks of the tile slots, [2] tiles relocated
    float alpha;                  // 0.5*dt/m_q (species.cpp:2305)
    float dt_dx, dt_dy;           // dt/dx (species.cpp:2140-2143)
    float q;                      // charge per particle
    float qnx, qny;               // q*dx/dt (species.cpp:2145-2148)
    int perx, pery;               // particle periodic flags
    int bc[4];                    // species::bc
    int min_slack;                // minimum free slots per tile after a repack
    float pool_frac;              // share of the free capacity kept as the pool at a repack (option "pool_fraction")
    float reloc_room;             // room given to a relocated tile, as a share of its count (option "relocation_room")
    float jscale;                 // fixed-point tile current: 2^k with |q| * jscale < 2^30
    double jscale_inv;            // 1 / jscale
};

// ---------------------------------------------------------------------------
// PTX helpers: bulk asynchronous copies (TMA, non-tensor form) and mbarriers.
// No multicast forms are used anywhere.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32( const void * p ) {
    return static_cast<uint32_t>( __cvta_generic_to_shared( p ) );
}

__device__ __forceinline__ void mbar_init( uint64_t * bar, uint32_t count ) {
    asm volatile( "mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"( smem_u32( bar ) ), "r"( count ) : "memory" );
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile( "fence.mbarrier_init.release.cluster;" ::: "memory" );
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile( "fence.proxy.async.shared::cta;" ::: "memory" );
}

__device__ __forceinline__ void mbar_arrive_expect_tx( uint64_t * bar, uint32_t bytes ) {
    asm volatile( "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                  :: "r"( smem_u32( bar ) ), "r"( bytes ) : "memory" );
}

// Non-blocking test of an mbarrier phase.
__device__ __forceinline__ bool mbar_test_wait_parity( uint64_t * bar, uint32_t parity ) {
    uint32_t ok;
    asm volatile( "{\n\t.reg .pred p;\n\t"
                  "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                  "selp.u32 %0, 1, 0, p;\n\t}"
                  : "=r"( ok ) : "r"( smem_u32( bar ) ), "r"( parity ) : "memory" );
    return ok != 0;
}

// Test of an mbarrier phase that may suspend the thread for a while (a
// hardware-chosen time) before it reports the phase incomplete.
__device__ __forceinline__ bool mbar_try_wait_parity( uint64_t * bar, uint32_t parity ) {
    uint32_t ok;
    asm volatile( "{\n\t.reg .pred p;\n\t"
                  "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                  "selp.u32 %0, 1, 0, p;\n\t}"
                  : "=r"( ok ) : "r"( smem_u32( bar ) ), "r"( parity ) : "memory" );
    return ok != 0;
}

// Global -> shared bulk copy completing on an mbarrier.  dst, src 16-byte
// aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s( void * dst, const void * src, uint32_t bytes, uint64_t * bar ) {
    asm volatile( "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                  :: "r"( smem_u32( dst ) ), "l"( src ), "r"( bytes ), "r"( smem_u32( bar ) ) : "memory" );
}

// Shared -> global bulk copy (bulk-group completion).
__device__ __forceinline__ void bulk_s2g( void * dst, const void * src, uint32_t bytes ) {
    asm volatile( "cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
                  :: "l"( dst ), "r"( smem_u32( src ) ), "r"( bytes ) : "memory" );
}

// Shared -> global bulk element-wise reduction: dst[i] += src[i] (f32, atomic per element).
__device__ __forceinline__ void bulk_s2g_add_f32( float * dst, const float * src, uint32_t bytes ) {
    asm volatile( "cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f32 [%0], [%1], %2;"
                  :: "l"( dst ), "r"( smem_u32( src ) ), "r"( bytes ) : "memory" );
}

__device__ __forceinline__ void bulk_commit() {
    asm volatile( "cp.async.bulk.commit_group;" ::: "memory" );
}

// Wait until the shared-memory sources of all committed bulk groups have been read.
__device__ __forceinline__ void bulk_wait_read_all() {
    asm volatile( "cp.async.bulk.wait_group.read 0;" ::: "memory" );
}

// Wait until all committed bulk groups are complete (writes visible).
__device__ __forceinline__ void bulk_wait_all() {
    asm volatile( "cp.async.bulk.wait_group 0;" ::: "memory" );
}

// Polls of a bounded wait by default: ~0.5 s.
constexpr int WAIT_LIMIT_DEFAULT = 1 << 22;

// Bounded wait on an mbarrier phase.  Gives up after `limit` polls, records
// ST_WAIT_TIMEOUT (when status is given) and returns false; never traps.  The
// first poll does not block (so that a limit of 1 tests the phase once), the
// later ones may.
__device__ __forceinline__ bool mbar_wait_bounded( uint64_t * bar, uint32_t parity, int * status,
                                                   int limit = WAIT_LIMIT_DEFAULT ) {
    for ( int i = 0; i < limit; i++ ) {
        if ( i == 0 ? mbar_test_wait_parity( bar, parity ) : mbar_try_wait_parity( bar, parity ) ) return true;
        if ( i > 16 ) __nanosleep( 128 );
    }
    if ( status ) atomicOr( status, ST_WAIT_TIMEOUT );
    return false;
}

// Bulk copies into shared memory complete on an mbarrier.  A CTA whose wait
// gave up must not compute on (or store) what has not arrived, and must not
// exit while its copies may still write its shared memory: every thread
// learns whether any thread gave up, and if so waits once more, with the
// default limit, for the copies to land.  Returns true when the CTA must
// skip its work and return.
__device__ __forceinline__ bool bulk_wait_or_abandon( uint64_t * bar, int * status, int limit ) {
    const bool ok = mbar_wait_bounded( bar, 0, status, limit );
    if ( !__syncthreads_or( !ok ) ) return false;
    mbar_wait_bounded( bar, 0, status, WAIT_LIMIT_DEFAULT );
    __syncthreads();
    return true;
}

// Tile-local cell index packing
__device__ __forceinline__ uint32_t pack_cell( int ix, int iy ) {
    return ( static_cast<uint32_t>( ix ) & 0xFFFFu ) | ( static_cast<uint32_t>( iy ) << 16 );
}
__device__ __forceinline__ int cell_x( uint32_t c ) { return static_cast<int>( static_cast<int16_t>( c & 0xFFFFu ) ); }
__device__ __forceinline__ int cell_y( uint32_t c ) { return static_cast<int>( static_cast<int16_t>( c >> 16 ) ); }

// Work item of the particle kernels: species, tile, chunk
struct Item { int sp; int tile; int chunk; int pad; };

// Phase-space deposit parameters (quantities 0 x, 1 y, 2 ux, 3 uy, 4 uz;
// q1 < 0 for a 1D phase space).  r = lower range bound in deposit units,
// rdx = bins per unit, norm = weight of one particle.
struct PhaSpec { int q0, q1, n0, n1; float r0, rdx0, r1, rdx1, norm; int smem; };

// Density injection rule of one species (Injector, density.cpp): which
// in-cell positions of a global cell range receive a particle.
struct InjRule {
    int type;                 // 1 uniform, 2 step, 3 slab, 4 sphere
    int diry;
    float a, b;               // step pos / slab begin,end (cells)
    float cx, cy, r2;         // sphere (simulation units)
    float dxx, dxy;
    int ppcx, ppcy;
    int range[4];             // x.lower, x.upper, y.lower, y.upper (global cells)
    int tx_limit;             // tiles processed along x (reference quirk for dir = y)
    const float * dyn;        // if set: a, b, cx computed on the device for the window's position
};

}  // namespace zb
