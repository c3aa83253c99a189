// fields.cu -- grid kernels of the em2d step for sm_100a: current guard-cell
// accumulation, Yee solver, E/B guard-cell exchange, physical boundaries,
// digital filters, moving-window shift and field energy.
//
// Compiled with -fmad=false like particles.cu; all field updates are
// deterministic (no atomics) and bit-identical to the reference for the same
// inputs.
#include "zpic_dev.cuh"

namespace zb {

struct TileItem { int run; int tile; };

// Guard cells are {1,2} on both axes for E, B and J (emf.cpp:31-33, current.cpp:24-26).
constexpr int GL = 1, GU = 2;

__device__ __forceinline__ int nbr( int v, int n, int periodic ) {
    if ( periodic ) { if ( v < 0 ) v += n; else if ( v >= n ) v -= n; return v; }
    return ( v >= 0 && v < n ) ? v : -1;
}

// ---------------------------------------------------------------------------
// Guard-cell resolution.
//
// grid::copy_to_gc (grid.h:253-354) is an x pass followed by a y pass.  The
// value a cell holds afterwards is the value of the cell found by first
// stepping into the y neighbour (if the cell is a y guard and the neighbour
// exists) and then, in that tile, into the x neighbour.  Sources are always
// cells this pass never writes, so one kernel can update guard cells in place.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void resolve_copy( const RunDev & R, int perx, int pery, int axes,
                                              int tx, int ty, int i, int j,
                                              int & stx, int & sty, int & si, int & sj ) {
    stx = tx; sty = ty; si = i; sj = j;
    if ( axes & 2 ) {
        if ( j < GL ) {
            const int n = nbr( ty - 1, R.nty, pery );
            if ( n >= 0 ) { sty = n; sj = j + R.nxy; }
        } else if ( j >= GL + R.nxy ) {
            const int n = nbr( ty + 1, R.nty, pery );
            if ( n >= 0 ) { sty = n; sj = j - R.nxy; }
        }
    }
    if ( axes & 1 ) {
        if ( i < GL ) {
            const int n = nbr( tx - 1, R.ntx, perx );
            if ( n >= 0 ) { stx = n; si = i + R.nxx; }
        } else if ( i >= GL + R.nxx ) {
            const int n = nbr( tx + 1, R.ntx, perx );
            if ( n >= 0 ) { stx = n; si = i - R.nxx; }
        }
    }
}

__device__ __forceinline__ const float * cellp( const float * g, const RunDev & R, int tx, int ty, int i, int j ) {
    return g + ( (size_t) ( ty * R.ntx + tx ) * R.tile_vol + j * R.extx + i ) * 3;
}

// x pass of grid::add_from_gc (grid.h:360-403) at one cell
__device__ __forceinline__ void add_x( const float * raw, const RunDev & R, int perx, int tx, int ty, int i, int j,
                                       float & a, float & b, float & c ) {
    const float * p = cellp( raw, R, tx, ty, i, j );
    a = p[0]; b = p[1]; c = p[2];
    if ( i >= GL && i < GL + GU ) {
        const int n = nbr( tx - 1, R.ntx, perx );
        if ( n >= 0 ) { const float * q = cellp( raw, R, n, ty, i + R.nxx, j ); a += q[0]; b += q[1]; c += q[2]; }
    }
    if ( i >= R.nxx && i < R.nxx + GL ) {
        const int n = nbr( tx + 1, R.ntx, perx );
        if ( n >= 0 ) { const float * q = cellp( raw, R, n, ty, i - R.nxx, j ); a += q[0]; b += q[1]; c += q[2]; }
    }
}

// add_from_gc (x pass, then y pass over the x-pass results; grid.h:405-445)
__device__ __forceinline__ void add_xy( const float * raw, const RunDev & R, int perx, int pery, int tx, int ty, int i, int j,
                                        float & a, float & b, float & c ) {
    add_x( raw, R, perx, tx, ty, i, j, a, b, c );
    if ( j >= GL && j < GL + GU ) {
        const int n = nbr( ty - 1, R.nty, pery );
        if ( n >= 0 ) { float p, q, r; add_x( raw, R, perx, tx, n, i, j + R.nxy, p, q, r ); a += p; b += q; c += r; }
    }
    if ( j >= R.nxy && j < R.nxy + GL ) {
        const int n = nbr( ty + 1, R.nty, pery );
        if ( n >= 0 ) { float p, q, r; add_x( raw, R, perx, tx, n, i, j - R.nxy, p, q, r ); a += p; b += q; c += r; }
    }
}

// The guard-cell copies run one thread per guard cell of every tile of the
// work list: thread gid handles guard cell gid % per of item gid / per, so
// the many small, independent copies of all tiles are in flight at once.
constexpr int GC_THREADS = 256;

// Guard cell g (row-major over the tile's guard region) -> tile cell (i, j):
// the GL bottom rows, the GU top rows, then the GL left and GU right cells of
// every interior row.
__device__ __forceinline__ void guard_cell( int g, const RunDev & R, int & i, int & j ) {
    const int bottom = GL * R.extx;
    if ( g < bottom ) { i = g % R.extx; j = g / R.extx; return; }
    g -= bottom;
    const int top = GU * R.extx;
    if ( g < top ) { i = g % R.extx; j = GL + R.nxy + g / R.extx; return; }
    g -= top;
    const int c = g % ( GL + GU );
    j = GL + g / ( GL + GU );
    i = c < GL ? c : R.nxx + c;
}

__device__ __forceinline__ int guard_count( const RunDev & R ) { return R.extx * R.exty - R.nxx * R.nxy; }

// Current::advance's add_from_gc + copy_to_gc (current.cpp:227-233) in one
// pass: Jdep (tile-local deposits) -> J (summed, guard cells refreshed).  One
// CTA per tile: each cell gathers up to nine contributions, and a tile's
// threads read neighbouring cells together (measured faster than one thread
// per cell of all tiles for this kernel, unlike the pure copies below).
__global__ void __launch_bounds__( 128 )
k_current_gc( const TileItem * __restrict__ items, const RunDev * __restrict__ runs )
{
    const TileItem it = items[ blockIdx.x ];
    const RunDev & R = runs[ it.run ];
    const int tx = it.tile % R.ntx, ty = it.tile / R.ntx;
    const int ncell = R.extx * R.exty;
    float * out = R.J + (size_t) it.tile * R.tile_vol * 3;
    for ( int c = threadIdx.x; c < ncell; c += blockDim.x ) {
        const int i = c % R.extx, j = c / R.extx;
        int stx, sty, si, sj;
        resolve_copy( R, R.cur_perx, R.cur_pery, 3, tx, ty, i, j, stx, sty, si, sj );
        float a, b, d;
        add_xy( R.Jdep, R, R.cur_perx, R.cur_pery, stx, sty, si, sj, a, b, d );
        out[3*c] = a; out[3*c+1] = b; out[3*c+2] = d;
    }
}

// the tile right of (tx, ty) for E and B, or -1
__device__ __forceinline__ int right_tile( const RunDev & R, int tx, int ty ) {
    const int n = nbr( tx + 1, R.ntx, R.emf_perx );
    return n >= 0 ? ty * R.ntx + n : -1;
}

// grid::copy_to_gc on E and B in place (axes: 1 x, 2 y, 3 both).
// bfix: after a Yee kernel that wrote its tile shifted one cell to the left
// (shift_out), B of every tile's new last interior column is the right
// neighbour's first interior column saved in bcol (where there is a right
// neighbour): the threads after the guard cells of a tile write it, and guard
// cells whose source is such a cell read it from bcol as well.
__global__ void __launch_bounds__( GC_THREADS )
k_emf_gc( const TileItem * __restrict__ items, int nitems, int per, const RunDev * __restrict__ runs, int axes,
          int bfix )
{
    const unsigned gid = blockIdx.x * blockDim.x + threadIdx.x;     // n * per < 2^31 (launcher)
    const int w = (int) ( gid / (unsigned) per ), g = (int) ( gid % (unsigned) per );
    if ( w >= nitems ) return;
    const TileItem it = items[w];
    const RunDev & R = runs[ it.run ];
    const int tx = it.tile % R.ntx, ty = it.tile / R.ntx;
    const int ng = guard_count( R );
    if ( g >= ng ) {
        const int row = g - ng;
        if ( !bfix || row >= R.nxy ) return;
        const int rn = right_tile( R, tx, ty );
        if ( rn < 0 ) return;
        const size_t dst = ( (size_t) it.tile * R.tile_vol + ( GL + row ) * R.extx + GL + R.nxx - 1 ) * 3;
        const float * b = R.bcol + ( (size_t) rn * R.nxy + row ) * 3;
        const float b0 = b[0], b1 = b[1], b2 = b[2];
        R.B[dst] = b0; R.B[dst + 1] = b1; R.B[dst + 2] = b2;
        return;
    }
    int i, j;
    guard_cell( g, R, i, j );
    int stx, sty, si, sj;
    resolve_copy( R, R.emf_perx, R.emf_pery, axes, tx, ty, i, j, stx, sty, si, sj );
    if ( stx == tx && sty == ty && si == i && sj == j ) return;
    const size_t dst = ( (size_t) it.tile * R.tile_vol + j * R.extx + i ) * 3;
    const float * e = cellp( R.E, R, stx, sty, si, sj );
    const float * b = cellp( R.B, R, stx, sty, si, sj );
    if ( bfix && si == GL + R.nxx - 1 && sj >= GL && sj < GL + R.nxy ) {
        const int rn = right_tile( R, stx, sty );
        if ( rn >= 0 ) b = R.bcol + ( (size_t) rn * R.nxy + sj - GL ) * 3;
    }
    const float e0 = e[0], e1 = e[1], e2 = e[2], b0 = b[0], b1 = b[1], b2 = b[2];
    R.E[dst] = e0; R.E[dst + 1] = e1; R.E[dst + 2] = e2;
    R.B[dst] = b0; R.B[dst + 1] = b1; R.B[dst + 2] = b2;
}

// J guard-cell refresh only (used after current filters): axes 1 x, 2 y
__global__ void __launch_bounds__( GC_THREADS )
k_cur_gc( const TileItem * __restrict__ items, int nitems, int per, const RunDev * __restrict__ runs, int axes )
{
    const unsigned gid = blockIdx.x * blockDim.x + threadIdx.x;     // n * per < 2^31 (launcher)
    const int w = (int) ( gid / (unsigned) per ), g = (int) ( gid % (unsigned) per );
    if ( w >= nitems ) return;
    const TileItem it = items[w];
    const RunDev & R = runs[ it.run ];
    if ( g >= guard_count( R ) ) return;
    const int tx = it.tile % R.ntx, ty = it.tile / R.ntx;
    int i, j;
    guard_cell( g, R, i, j );
    int stx, sty, si, sj;
    resolve_copy( R, R.cur_perx, R.cur_pery, axes, tx, ty, i, j, stx, sty, si, sj );
    if ( stx == tx && sty == ty && si == i && sj == j ) return;
    const size_t dst = ( (size_t) it.tile * R.tile_vol + j * R.extx + i ) * 3;
    const float * q = cellp( R.J, R, stx, sty, si, sj );
    const float q0 = q[0], q1 = q[1], q2 = q[2];
    R.J[dst] = q0; R.J[dst + 1] = q1; R.J[dst + 2] = q2;
}

// ---------------------------------------------------------------------------
// Yee solver (emf.cpp:513-580): per tile, E, B and J tiles staged into shared
// memory with bulk asynchronous copies; B half step over [-1,nx], E step with
// J over [0,nx+1], B half step; E and B tiles stored back with bulk copies.
// The raw deposit buffer of the tile is cleared for the next step.
// ---------------------------------------------------------------------------
constexpr int YEE_THREADS = 256;

__device__ __forceinline__ void yee_b_smem( const float * E, float * B, const RunDev & R, float dtx, float dty ) {
    const int ys = R.extx;
    const int w = R.nxx + 2, h = R.nxy + 2;
    for ( int c = threadIdx.x; c < w * h; c += blockDim.x ) {
        const int ix = c % w - 1, iy = c / w - 1;
        const int k = 3 * ( ix + iy * ys ), kx = 3 * ( ix + 1 + iy * ys ), ky = 3 * ( ix + ( iy + 1 ) * ys );
        B[k + 0] += ( -dty * ( E[ky + 2] - E[k + 2] ) );
        B[k + 1] += (  dtx * ( E[kx + 2] - E[k + 2] ) );
        B[k + 2] += ( -dtx * ( E[kx + 1] - E[k + 1] ) + dty * ( E[ky + 0] - E[k + 0] ) );
    }
}

__device__ __forceinline__ void yee_e_smem( float * E, const float * B, const float * J, const RunDev & R,
                                            float dtx, float dty, float dt, int with_j ) {
    const int ys = R.extx;
    const int w = R.nxx + 2, h = R.nxy + 2;
    for ( int c = threadIdx.x; c < w * h; c += blockDim.x ) {
        const int ix = c % w, iy = c / w;
        const int k = 3 * ( ix + iy * ys ), kx = 3 * ( ix - 1 + iy * ys ), ky = 3 * ( ix + ( iy - 1 ) * ys );
        if ( with_j ) {
            E[k + 0] += ( +dty * ( B[k + 2] - B[ky + 2] ) ) - dt * J[k + 0];
            E[k + 1] += ( -dtx * ( B[k + 2] - B[kx + 2] ) ) - dt * J[k + 1];
            E[k + 2] += ( +dtx * ( B[k + 1] - B[kx + 1] ) - dty * ( B[k + 0] - B[ky + 0] ) ) - dt * J[k + 2];
        } else {
            E[k + 0] += ( +dty * ( B[k + 2] - B[ky + 2] ) );
            E[k + 1] += ( -dtx * ( B[k + 2] - B[kx + 2] ) );
            E[k + 2] += ( +dtx * ( B[k + 1] - B[kx + 1] ) - dty * ( B[k + 0] - B[ky + 0] ) );
        }
    }
}

__global__ void __launch_bounds__( YEE_THREADS )
k_yee( const TileItem * __restrict__ items, const RunDev * __restrict__ runs, int with_j, int j_raw, int clear_jdep,
       int shift_out )
{
    extern __shared__ __align__( 16 ) unsigned char smem_raw[];
    const TileItem it = items[ blockIdx.x ];
    const RunDev & R = runs[ it.run ];
    const int tv = R.tile_vol;
    float * sE = reinterpret_cast<float *>( smem_raw );
    float * sB = sE + 3 * tv;
    float * sJ = sB + 3 * tv;
    uint64_t * bar = reinterpret_cast<uint64_t *>( sJ + 3 * tv );
    const size_t toff = (size_t) it.tile * 3 * tv;
    const uint32_t bytes = 12u * tv;
    const float * Jsrc = j_raw ? R.Jdep : R.J;

    if ( threadIdx.x == 0 ) { mbar_init( bar, 1 ); fence_mbar_init(); }
    __syncthreads();
    if ( threadIdx.x == 0 ) {
        mbar_arrive_expect_tx( bar, with_j ? 3 * bytes : 2 * bytes );
        bulk_g2s( sE, R.E + toff, bytes, bar );
        bulk_g2s( sB, R.B + toff, bytes, bar );
        if ( with_j ) bulk_g2s( sJ, Jsrc + toff, bytes, bar );
    }
    // an expired wait: no field update and no stores for this tile
    if ( bulk_wait_or_abandon( bar, R.status, R.wait_limit ) ) return;

    float * E0 = sE + 3 * R.gc_off;
    float * B0 = sB + 3 * R.gc_off;
    const float * J0 = sJ + 3 * R.gc_off;
    yee_b_smem( E0, B0, R, R.dtx2, R.dty2 );
    __syncthreads();
    yee_e_smem( E0, B0, J0, R, R.dtx, R.dty, R.dt, with_j );
    __syncthreads();
    yee_b_smem( E0, B0, R, R.dtx2, R.dty2 );
    __syncthreads();

    const float * outE = sE, * outB = sB;
    if ( shift_out ) {
        // a window shift (grid::x_shift_left(1)) follows at once: the tile is
        // stored one cell to the left, the last cell of every row cleared --
        // E shifted into the current tile's place (free after the E step),
        // then B into E's.  The new last interior column is the first upper
        // guard column: E there is this kernel's own update of it, bit for bit
        // the right neighbour's (same inputs, same arithmetic); B there would
        // need E one column further out, so the first interior column of B is
        // saved (bcol) and the guard refresh that follows (k_emf_gc, bfix)
        // puts the right neighbour's in place, refreshing every guard cell.
        float * dst = R.bcol + (size_t) it.tile * R.nxy * 3;
        for ( int q = threadIdx.x; q < 3 * R.nxy; q += blockDim.x ) dst[q] = B0[ 3 * ( ( q / 3 ) * R.extx ) + q % 3 ];
        const int ys = R.extx, nc = 3 * R.extx * R.exty;
        float * sT = sJ;
        for ( int e = threadIdx.x; e < 3 * tv; e += blockDim.x )
            sT[e] = e < nc ? ( ( ( e / 3 ) % ys < ys - 1 ) ? sE[ e + 3 ] : 0.0f ) : sE[e];
        __syncthreads();
        for ( int e = threadIdx.x; e < 3 * tv; e += blockDim.x )
            sE[e] = e < nc ? ( ( ( e / 3 ) % ys < ys - 1 ) ? sB[ e + 3 ] : 0.0f ) : sB[e];
        __syncthreads();
        outE = sT; outB = sE;
    }
    if ( threadIdx.x == 0 ) {
        fence_proxy_async_smem();
        bulk_s2g( R.E + toff, outE, bytes );
        bulk_s2g( R.B + toff, outB, bytes );
        bulk_commit();
    }
    if ( clear_jdep ) {
        float4 * z = reinterpret_cast<float4 *>( R.Jdep + toff );
        for ( int i = threadIdx.x; i < 3 * tv / 4; i += blockDim.x ) z[i] = make_float4( 0.f, 0.f, 0.f, 0.f );
    }
    // the shared-memory sources read; the stores complete before the kernel does
    if ( threadIdx.x == 0 ) bulk_wait_read_all();
}

// ---------------------------------------------------------------------------
// Physical boundaries (rare paths): PEC/PMC fields (emf.cpp:207-410),
// reflecting current (current.cpp:53-160).  One thread per boundary row.
// ---------------------------------------------------------------------------
__global__ void k_emf_bc( const RunDev * __restrict__ runs, int run, int axis )
{
    const RunDev & R = runs[run];
    const int pec = 2, pmc = 3;
    const int ys = R.extx;
    if ( axis == 0 ) {
        // tiles (0, ty) and (ntx-1, ty); reference loops tx in {0, ntx-1}
        const int k = blockIdx.x * blockDim.x + threadIdx.x;
        const int nrow = R.exty;
        if ( k >= 2 * R.nty * nrow ) return;
        const int side = k / ( R.nty * nrow ), rem = k % ( R.nty * nrow );
        const int ty = rem / nrow, idx = rem % nrow;
        const int tx = side ? R.ntx - 1 : 0;
        if ( side == 1 && R.ntx == 1 ) return;   // tile 0 visited twice; the lower rule is idempotent
        float * E = R.E + ( (size_t) ( ty * R.ntx + tx ) * R.tile_vol + GL ) * 3;
        float * B = R.B + ( (size_t) ( ty * R.ntx + tx ) * R.tile_vol + GL ) * 3;
        const int iy = idx * ys;
        const int nx = R.nxx;
#define e( c, k ) E[ 3 * ( c ) + k ]
#define b( c, k ) B[ 3 * ( c ) + k ]
        if ( tx == 0 ) {
            if ( R.emf_bc[0] == pmc ) {
                e( -1 + iy, 0 ) = -e( 0 + iy, 0 ); e( -1 + iy, 1 ) = e( 1 + iy, 1 ); e( -1 + iy, 2 ) = e( 1 + iy, 2 );
                b( -1 + iy, 0 ) = b( 1 + iy, 0 ); b( -1 + iy, 1 ) = -b( 0 + iy, 1 ); b( -1 + iy, 2 ) = -b( 0 + iy, 2 );
            } else if ( R.emf_bc[0] == pec ) {
                e( -1 + iy, 0 ) = e( 0 + iy, 0 ); e( -1 + iy, 1 ) = -e( 1 + iy, 1 ); e( -1 + iy, 2 ) = -e( 1 + iy, 2 );
                e( 0 + iy, 1 ) = 0; e( 0 + iy, 2 ) = 0;
                b( -1 + iy, 0 ) = -b( 1 + iy, 0 ); b( -1 + iy, 1 ) = b( 0 + iy, 1 ); b( -1 + iy, 2 ) = b( 0 + iy, 2 );
                b( 0 + iy, 0 ) = 0;
            }
        } else {
            if ( R.emf_bc[1] == pmc ) {
                e( nx + iy, 0 ) = -e( nx - 1 + iy, 0 );
                e( nx + 1 + iy, 0 ) = -e( nx - 2 + iy, 0 ); e( nx + 1 + iy, 1 ) = e( nx - 1 + iy, 1 ); e( nx + 1 + iy, 2 ) = e( nx - 1 + iy, 2 );
                b( nx + iy, 1 ) = -b( nx - 1 + iy, 1 ); b( nx + iy, 2 ) = -b( nx - 1 + iy, 2 );
                b( nx + 1 + iy, 0 ) = b( nx - 1 + iy, 0 ); b( nx + 1 + iy, 1 ) = -b( nx - 2 + iy, 1 ); b( nx + 1 + iy, 2 ) = -b( nx - 2 + iy, 2 );
            } else if ( R.emf_bc[1] == pec ) {
                e( nx + iy, 0 ) = e( nx - 1 + iy, 0 ); e( nx + iy, 1 ) = 0; e( nx + iy, 2 ) = 0;
                e( nx + 1 + iy, 0 ) = e( nx - 2 + iy, 0 ); e( nx + 1 + iy, 1 ) = -e( nx - 1 + iy, 1 ); e( nx + 1 + iy, 2 ) = -e( nx - 1 + iy, 2 );
                b( nx + iy, 0 ) = 0; b( nx + iy, 1 ) = b( nx - 1 + iy, 1 ); b( nx + iy, 2 ) = b( nx - 1 + iy, 2 );
                b( nx + 1 + iy, 0 ) = -b( nx - 1 + iy, 0 ); b( nx + 1 + iy, 1 ) = b( nx - 2 + iy, 1 ); b( nx + 1 + iy, 2 ) = b( nx - 2 + iy, 2 );
            }
        }
    } else {
        const int k = blockIdx.x * blockDim.x + threadIdx.x;
        const int ncol = R.extx;
        if ( k >= 2 * R.ntx * ncol ) return;
        const int side = k / ( R.ntx * ncol ), rem = k % ( R.ntx * ncol );
        const int tx = rem / ncol, ix = rem % ncol;
        const int ty = side ? R.nty - 1 : 0;
        if ( side == 1 && R.nty == 1 ) return;
        float * E = R.E + ( (size_t) ( ty * R.ntx + tx ) * R.tile_vol + GL * ys ) * 3;
        float * B = R.B + ( (size_t) ( ty * R.ntx + tx ) * R.tile_vol + GL * ys ) * 3;
        // The reference indexes a few upper-y source rows with nx.x instead of
        // nx.y (emf.cpp:377-399).  Same rows for square tiles; for other tiles
        // those rows would lie outside the tile block, so nx.y is used there.
        const int ny = R.nxy, nx = ( R.nxx + 1 < R.exty - GL ) ? R.nxx : R.nxy;
        if ( ty == 0 ) {
            if ( R.emf_bc[2] == pmc ) {
                e( ix - ys, 0 ) = e( ix + ys, 0 ); e( ix - ys, 1 ) = -e( ix, 1 ); e( ix - ys, 2 ) = e( ix + ys, 2 );
                b( ix - ys, 0 ) = -b( ix, 0 ); b( ix - ys, 1 ) = b( ix + ys, 1 ); b( ix - ys, 2 ) = -b( ix, 2 );
            } else if ( R.emf_bc[2] == pec ) {
                e( ix - ys, 0 ) = -e( ix + ys, 0 ); e( ix - ys, 1 ) = e( ix, 1 ); e( ix - ys, 2 ) = -e( ix + ys, 2 );
                e( ix, 0 ) = 0; e( ix, 2 ) = 0;
                b( ix - ys, 0 ) = b( ix, 0 ); b( ix - ys, 1 ) = -b( ix + ys, 1 ); b( ix - ys, 2 ) = b( ix, 2 );
                b( ix, 1 ) = 0;
            }
        } else {
            if ( R.emf_bc[3] == pmc ) {
                e( ix + ny * ys, 1 ) = -e( ix + ( ny - 1 ) * ys, 1 );
                e( ix + ( ny + 1 ) * ys, 0 ) = e( ix + ( ny - 1 ) * ys, 0 );
                e( ix + ( ny + 1 ) * ys, 1 ) = -e( ix + ( ny - 2 ) * ys, 1 );
                e( ix + ( ny + 1 ) * ys, 2 ) = e( ix + ( ny - 1 ) * ys, 2 );
                b( ix + ny * ys, 0 ) = -b( ix + ( ny - 1 ) * ys, 0 );
                b( ix + ny * ys, 2 ) = -b( ix + ( ny - 1 ) * ys, 2 );
                b( ix + ( ny + 1 ) * ys, 0 ) = -b( ix + ( nx - 2 ) * ys, 0 );
                b( ix + ( ny + 1 ) * ys, 1 ) = b( ix + ( nx - 1 ) * ys, 1 );
                b( ix + ( ny + 1 ) * ys, 2 ) = -b( ix + ( nx - 2 ) * ys, 2 );
            } else if ( R.emf_bc[3] == pec ) {
                e( ix + ny * ys, 0 ) = 0;
                e( ix + ny * ys, 1 ) = e( ix + ( ny - 1 ) * ys, 1 );
                e( ix + ny * ys, 2 ) = 0;
                e( ix + ( ny + 1 ) * ys, 0 ) = -e( ix + ( nx - 1 ) * ys, 0 );
                e( ix + ( ny + 1 ) * ys, 1 ) = e( ix + ( nx - 2 ) * ys, 1 );
                e( ix + ( ny + 1 ) * ys, 2 ) = -e( ix + ( nx - 1 ) * ys, 2 );
                b( ix + ny * ys, 0 ) = b( ix + ( ny - 1 ) * ys, 0 );
                b( ix + ny * ys, 1 ) = 0;
                b( ix + ny * ys, 2 ) = b( ix + ( ny - 1 ) * ys, 2 );
                b( ix + ( ny + 1 ) * ys, 0 ) = b( ix + ( ny - 2 ) * ys, 0 );
                b( ix + ( ny + 1 ) * ys, 1 ) = -b( ix + ( ny - 1 ) * ys, 1 );
                b( ix + ( ny + 1 ) * ys, 2 ) = b( ix + ( ny - 2 ) * ys, 2 );
            }
        }
#undef e
#undef b
    }
}

__global__ void k_cur_bc( const RunDev * __restrict__ runs, int run, int axis )
{
    const RunDev & R = runs[run];
    const int refl = 2;
    const int ys = R.extx;
#define j( c, k ) J[ 3 * ( c ) + k ]
    if ( axis == 0 ) {
        const int k = blockIdx.x * blockDim.x + threadIdx.x;
        const int nrow = R.exty;
        if ( k >= 2 * R.nty * nrow ) return;
        const int side = k / ( R.nty * nrow ), rem = k % ( R.nty * nrow );
        const int ty = rem / nrow, idx = rem % nrow;
        const int tx = side ? R.ntx - 1 : 0;
        if ( side == 1 && R.ntx == 1 ) return;
        float * J = R.J + ( (size_t) ( ty * R.ntx + tx ) * R.tile_vol + GL ) * 3;
        const int iy = idx * ys, nx = R.nxx;
        if ( tx == 0 ) {
            if ( R.cur_bc[0] == refl ) {
                const float jx0 = -j( -1 + iy, 0 ) + j( 0 + iy, 0 );
                const float jy1 = j( -1 + iy, 1 ) + j( 1 + iy, 1 );
                const float jz1 = j( -1 + iy, 2 ) + j( 1 + iy, 2 );
                j( -1 + iy, 0 ) = j( 0 + iy, 0 ) = jx0;
                j( -1 + iy, 1 ) = j( 1 + iy, 1 ) = jy1;
                j( -1 + iy, 2 ) = j( 1 + iy, 2 ) = jz1;
            }
        } else {
            if ( R.cur_bc[1] == refl ) {
                const float jx0 = j( nx - 1 + iy, 0 ) - j( nx + iy, 0 );
                const float jy1 = j( nx - 1 + iy, 1 ) + j( nx + 1 + iy, 1 );
                const float jz1 = j( nx - 1 + iy, 2 ) + j( nx + 1 + iy, 2 );
                j( nx - 1 + iy, 0 ) = j( nx + iy, 0 ) = jx0;
                j( nx - 1 + iy, 1 ) = j( nx + 1 + iy, 1 ) = jy1;
                j( nx - 1 + iy, 2 ) = j( nx + 1 + iy, 2 ) = jz1;
            }
        }
    } else {
        const int k = blockIdx.x * blockDim.x + threadIdx.x;
        const int ncol = R.extx;
        if ( k >= 2 * R.ntx * ncol ) return;
        const int side = k / ( R.ntx * ncol ), rem = k % ( R.ntx * ncol );
        const int tx = rem / ncol, ix = rem % ncol;
        const int ty = side ? R.nty - 1 : 0;
        if ( side == 1 && R.nty == 1 ) return;
        float * J = R.J + ( (size_t) ( ty * R.ntx + tx ) * R.tile_vol + GL * ys ) * 3;
        const int ny = R.nxy;
        if ( ty == 0 ) {
            if ( R.cur_bc[2] == refl ) {
                const float jx1 = j( ix - ys, 0 ) + j( ix + ys, 0 );
                const float jy0 = -j( ix - ys, 1 ) + j( ix, 1 );
                const float jz1 = j( ix - ys, 2 ) + j( ix + ys, 2 );
                j( ix - ys, 0 ) = j( ix + ys, 0 ) = jx1;
                j( ix - ys, 1 ) = j( ix, 1 ) = jy0;
                j( ix - ys, 2 ) = j( ix + ys, 2 ) = jz1;
            }
        } else {
            if ( R.cur_bc[3] == refl ) {
                const float jx1 = j( ix + ( ny - 1 ) * ys, 0 ) + j( ix + ( ny + 1 ) * ys, 0 );
                const float jy0 = j( ix + ( ny - 1 ) * ys, 1 ) - j( ix + ny * ys, 1 );
                const float jz1 = j( ix + ( ny - 1 ) * ys, 2 ) + j( ix + ( ny + 1 ) * ys, 2 );
                j( ix + ( ny - 1 ) * ys, 0 ) = j( ix + ( ny + 1 ) * ys, 0 ) = jx1;
                j( ix + ( ny - 1 ) * ys, 1 ) = j( ix + ny * ys, 1 ) = jy0;
                j( ix + ( ny - 1 ) * ys, 2 ) = j( ix + ( ny + 1 ) * ys, 2 ) = jz1;
            }
        }
    }
#undef j
}

// 3-point convolution along x or y on one grid (grid.h:495-593); interior
// columns (x) for all rows, or interior rows (y) for all columns.
__global__ void __launch_bounds__( 128 )
k_kernel3( const TileItem * __restrict__ items, const RunDev * __restrict__ runs, int which, int diry,
           float a, float b, float c )
{
    extern __shared__ float sA[];
    const TileItem it = items[ blockIdx.x ];
    const RunDev & R = runs[ it.run ];
    float * g = ( which == 0 ? R.E : which == 1 ? R.B : R.J ) + (size_t) it.tile * R.tile_vol * 3;
    const int n = 3 * R.tile_vol;
    for ( int i = threadIdx.x; i < n; i += blockDim.x ) sA[i] = g[i];
    __syncthreads();
    const int ys = R.extx;
    if ( !diry ) {
        const int w = R.nxx, h = R.exty;
        for ( int q = threadIdx.x; q < w * h; q += blockDim.x ) {
            const int ix = GL + q % w, iy = q / w;
            for ( int k = 0; k < 3; k++ )
                g[ 3 * ( iy * ys + ix ) + k ] = sA[ 3 * ( iy * ys + ix - 1 ) + k ] * a +
                                                sA[ 3 * ( iy * ys + ix ) + k ] * b +
                                                sA[ 3 * ( iy * ys + ix + 1 ) + k ] * c;
        }
    } else {
        const int w = R.extx, h = R.nxy;
        for ( int q = threadIdx.x; q < w * h; q += blockDim.x ) {
            const int ix = q % w, iy = GL + q / w;
            for ( int k = 0; k < 3; k++ )
                g[ 3 * ( iy * ys + ix ) + k ] = sA[ 3 * ( ( iy - 1 ) * ys + ix ) + k ] * a +
                                                sA[ 3 * ( iy * ys + ix ) + k ] * b +
                                                sA[ 3 * ( ( iy + 1 ) * ys + ix ) + k ] * c;
        }
    }
}

// grid::x_shift_left(1) data motion on E and B (grid.h:455-485); the x guard
// refresh follows as a separate k_emf_gc( axes = 1 ) launch.  Both fields'
// tile blocks are staged in shared memory with 16-byte loads in one pass
// (3 tile_vol floats per field, a multiple of 4), then written back shifted
// by one cell, the last cell of every row cleared.
constexpr int SHIFT_THREADS = 256;

__global__ void __launch_bounds__( SHIFT_THREADS )
k_shift_left( const TileItem * __restrict__ items, const RunDev * __restrict__ runs )
{
    extern __shared__ __align__( 16 ) float sA[];   // [E block][B block]
    const TileItem it = items[ blockIdx.x ];
    const RunDev & R = runs[ it.run ];
    const int n = 3 * R.tile_vol, n4 = n >> 2;
    float * gE = R.E + (size_t) it.tile * n;
    float * gB = R.B + (size_t) it.tile * n;
#pragma unroll 4
    for ( int v = threadIdx.x; v < 2 * n4; v += SHIFT_THREADS ) {
        const float4 * src = reinterpret_cast<const float4 *>( v < n4 ? gE : gB );
        reinterpret_cast<float4 *>( sA )[v] = src[ v < n4 ? v : v - n4 ];
    }
    __syncthreads();
    const int ys = R.extx, nc = 3 * R.extx * R.exty;
#pragma unroll 4
    for ( int f = threadIdx.x; f < 2 * nc; f += SHIFT_THREADS ) {
        const int fld = f >= nc, e = f - fld * nc;    // float e of cell e / 3 in the field's block
        const int ix = ( e / 3 ) % ys;
        ( fld ? gB : gE )[e] = ( ix < ys - 1 ) ? sA[ fld * n + e + 3 ] : 0.0f;
    }
}

// EMF::get_energy (emf.cpp:662-713): per tile, six FP64 sums of the FP32
// squares over the reference's loop range (note its inner bound nx.y).
__global__ void k_field_energy( const RunDev * __restrict__ runs, int run, double * __restrict__ out, int ntiles )
{
    const RunDev & R = runs[run];
    const int lane = threadIdx.x & 31;
    const int t = blockIdx.x * ( blockDim.x >> 5 ) + ( threadIdx.x >> 5 );      // a warp per tile
    if ( t >= ntiles ) return;
    // inner bound nx.y as in the reference; limited to the tile row (ext_x - 1
    // cells from x = 0) where nx.y exceeds it
    const int ixmax = min( R.nxy, R.extx - GL );
    const int ncell = R.nxy * ixmax;
    const float * e = R.E + ( (size_t) t * R.tile_vol + R.gc_off ) * 3;
    const float * b = R.B + ( (size_t) t * R.tile_vol + R.gc_off ) * 3;
    // each term v * v in FP32, summed in FP64 (emf.cpp:662-713); lanes take
    // every 32nd cell, then a fixed-order warp tree
    double s[6] = { 0.0, 0.0, 0.0, 0.0, 0.0, 0.0 };
    for ( int c = lane; c < ncell; c += 32 ) {
        const int iy = c / ixmax, ix = c - iy * ixmax;
        const int o = 3 * ( iy * R.extx + ix );
#pragma unroll
        for ( int k = 0; k < 3; k++ ) {
            const float v = e[ o + k ], w = b[ o + k ];
            s[k] += v * v;
            s[3 + k] += w * w;
        }
    }
#pragma unroll
    for ( int k = 0; k < 6; k++ ) {
#pragma unroll
        for ( int d = 16; d > 0; d >>= 1 ) s[k] += __shfl_down_sync( 0xffffffffu, s[k], d );
        if ( lane == 0 ) out[ 6 * t + k ] = s[k];
    }
}

// Adds a tiled grid: dst += src over whole tile blocks (Laser::Pulse::add, laser.h:85-99)
__global__ void k_grid_add( float * __restrict__ dst, const float * __restrict__ src, size_t n )
{
    for ( size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x )
        dst[i] += src[i];
}

// Scalar charge grid (guard cells {0,1}): add_from_gc then gather to a dense grid.
__global__ void k_charge_finish( const float * __restrict__ raw, float * __restrict__ out,
                                 int ntx, int nty, int nxx, int nxy, int cextx, int cvol, int perx, int pery )
{
    const int gx = blockIdx.x * blockDim.x + threadIdx.x;
    const int gy = blockIdx.y;
    if ( gx >= ntx * nxx ) return;
    const int tx = gx / nxx, ty = gy / nxy, i = gx % nxx, j = gy % nxy;
    // x pass: local[nx.x + i] += x_upper[i] (gc.x.lower = 0, gc.x.upper = 1)
    auto at = [&]( int ttx, int tty, int ii, int jj ) { return raw[ (size_t) ( tty * ntx + ttx ) * cvol + jj * cextx + ii ]; };
    auto ax = [&]( int ttx, int tty, int ii, int jj ) {
        float v = at( ttx, tty, ii, jj );
        if ( ii < 1 ) {                         // rows/cols [gc.x.lower, gc.x.lower+gc.x.upper) = [0,1)
            const int n = perx ? ( ttx - 1 + ntx ) % ntx : ttx - 1;
            if ( n >= 0 ) v += at( n, tty, ii + nxx, jj );
        }
        return v;
    };
    float v = ax( tx, ty, i, j );
    if ( j < 1 ) {
        const int n = pery ? ( ty - 1 + nty ) % nty : ty - 1;
        if ( n >= 0 ) v += ax( tx, n, i, j + nxy );
    }
    out[ (size_t) gy * ntx * nxx + gx ] = v;
}

// Dense gather of one component of a vec3 grid (vec3grid.h:76-205)
__global__ void k_grid_gather( const float * __restrict__ g, float * __restrict__ out, int fc,
                               int ntx, int nxx, int nxy, int extx, int gc_off, int tile_vol, int dimx )
{
    const int gx = blockIdx.x * blockDim.x + threadIdx.x;
    const int gy = blockIdx.y;
    if ( gx >= dimx ) return;
    const int tx = gx / nxx, ty = gy / nxy, i = gx % nxx, j = gy % nxy;
    out[ (size_t) gy * dimx + gx ] = g[ ( (size_t) ( ty * ntx + tx ) * tile_vol + gc_off + j * extx + i ) * 3 + fc ];
}

}  // namespace zb

namespace zb {

size_t yee_smem_bytes( int tile_vol ) { return (size_t) 9 * tile_vol * sizeof( float ) + 16; }

static unsigned gc_blocks( int n, int per ) {
    return (unsigned) ( ( (long long) n * per + GC_THREADS - 1 ) / GC_THREADS );
}
static bool gc_fits( int n, int per ) { return (long long) n * per < ( 1LL << 31 ) - GC_THREADS; }
// per: guard cells of the largest tile of the list (unused by the current sum)
cudaError_t launch_current_gc( cudaStream_t st, const TileItem * items, int n, const RunDev * runs, int ) {
    if ( n > 0 ) k_current_gc<<< n, 128, 0, st >>>( items, runs );
    return cudaGetLastError();
}
cudaError_t launch_emf_gc( cudaStream_t st, const TileItem * items, int n, const RunDev * runs, int axes, int per,
                           int bfix_rows ) {
    per += bfix_rows;
    if ( !gc_fits( n, per ) ) return cudaErrorInvalidConfiguration;
    if ( n > 0 ) k_emf_gc<<< gc_blocks( n, per ), GC_THREADS, 0, st >>>( items, n, per, runs, axes, bfix_rows > 0 );
    return cudaGetLastError();
}
cudaError_t launch_cur_gc( cudaStream_t st, const TileItem * items, int n, const RunDev * runs, int axes, int per ) {
    if ( !gc_fits( n, per ) ) return cudaErrorInvalidConfiguration;
    if ( n > 0 ) k_cur_gc<<< gc_blocks( n, per ), GC_THREADS, 0, st >>>( items, n, per, runs, axes );
    return cudaGetLastError();
}
cudaError_t launch_yee( cudaStream_t st, const TileItem * items, int n, const RunDev * runs,
                        int with_j, int j_raw, int clear_jdep, int max_tile_vol, int shift_out ) {
    const size_t smem = yee_smem_bytes( max_tile_vol );
    if ( smem > 48 * 1024 ) cudaFuncSetAttribute( (const void *) k_yee, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem );
    if ( n > 0 ) k_yee<<< n, YEE_THREADS, smem, st >>>( items, runs, with_j, j_raw, clear_jdep, shift_out );
    return cudaGetLastError();
}
cudaError_t launch_emf_bc( cudaStream_t st, const RunDev * runs, int run, int axis, int nthreads ) {
    if ( nthreads > 0 ) k_emf_bc<<< ( nthreads + 127 ) / 128, 128, 0, st >>>( runs, run, axis );
    return cudaGetLastError();
}
cudaError_t launch_cur_bc( cudaStream_t st, const RunDev * runs, int run, int axis, int nthreads ) {
    if ( nthreads > 0 ) k_cur_bc<<< ( nthreads + 127 ) / 128, 128, 0, st >>>( runs, run, axis );
    return cudaGetLastError();
}
cudaError_t launch_kernel3( cudaStream_t st, const TileItem * items, int n, const RunDev * runs, int which, int diry,
                            float a, float b, float c, int max_tile_vol ) {
    const size_t smem = (size_t) 3 * max_tile_vol * sizeof( float );
    if ( smem > 48 * 1024 ) cudaFuncSetAttribute( (const void *) k_kernel3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem );
    if ( n > 0 ) k_kernel3<<< n, 128, smem, st >>>( items, runs, which, diry, a, b, c );
    return cudaGetLastError();
}
cudaError_t launch_shift_left( cudaStream_t st, const TileItem * items, int n, const RunDev * runs, int max_tile_vol ) {
    const size_t smem = (size_t) 6 * max_tile_vol * sizeof( float );
    if ( smem > 48 * 1024 ) cudaFuncSetAttribute( (const void *) k_shift_left, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem );
    if ( n > 0 ) k_shift_left<<< n, SHIFT_THREADS, smem, st >>>( items, runs );
    return cudaGetLastError();
}
cudaError_t launch_field_energy( cudaStream_t st, const RunDev * runs, int run, int ntiles, double * out ) {
    k_field_energy<<< ( ntiles + 7 ) / 8, 256, 0, st >>>( runs, run, out, ntiles );
    return cudaGetLastError();
}
cudaError_t launch_grid_add( cudaStream_t st, float * dst, const float * src, size_t n ) {
    k_grid_add<<< 1184, 256, 0, st >>>( dst, src, n );
    return cudaGetLastError();
}
cudaError_t launch_charge_finish( cudaStream_t st, const float * raw, float * out, int ntx, int nty, int nxx, int nxy,
                                  int cextx, int cvol, int perx, int pery ) {
    dim3 g( ( ntx * nxx + 127 ) / 128, nty * nxy );
    k_charge_finish<<< g, 128, 0, st >>>( raw, out, ntx, nty, nxx, nxy, cextx, cvol, perx, pery );
    return cudaGetLastError();
}
cudaError_t launch_grid_gather( cudaStream_t st, const float * g, float * out, int fc, int ntx, int nty, int nxx, int nxy,
                                int extx, int gc_off, int tile_vol ) {
    dim3 gr( ( ntx * nxx + 127 ) / 128, nty * nxy );
    k_grid_gather<<< gr, 128, 0, st >>>( g, out, fc, ntx, nxx, nxy, extx, gc_off, tile_vol, ntx * nxx );
    return cudaGetLastError();
}

}  // namespace zb
