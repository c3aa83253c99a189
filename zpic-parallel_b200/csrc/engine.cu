// engine.cu -- host engine and C-ABI of libzpic_b200.so.
//
// A zpic_sim owns one simulation's device state (E, B, J, raw deposits,
// species particle slots and sort scratch) and a CUDA stream.  Every step is
// a fixed sequence of launches over work lists of (species, tile, chunk) and
// (run, tile) items; a zpic_batch builds the same lists over many
// simulations so that each phase of all of them is one launch.  Repeated
// steps are captured once in a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "zpic_b200.h"
#include "zpic_dev.cuh"
#include "host_init.h"

namespace zb {
struct TileItem { int run; int tile; };
size_t particle_smem_bytes( int tile_vol, int jacc );
size_t yee_smem_bytes( int tile_vol );
cudaError_t launch_particles( cudaStream_t, int, int, int, const Item *, int, const SpDev *, const RunDev *, const int *,
                              int, int, int );
cudaError_t launch_sort( cudaStream_t, const Item *, int, const SpDev *, const int *, int, const RunDev *, int, int * );
cudaError_t launch_inject( cudaStream_t, int, int, int, int, int, const SpDev *, const RunDev *, const InjRule &, int );
cudaError_t launch_inj_dyn( cudaStream_t, float *, unsigned *, int, float, float, float, double );
cudaError_t launch_pack( cudaStream_t, int, int, const SpDev *, const int *, int2 *, float2 *, float * );
cudaError_t launch_unpack( cudaStream_t, int, int, int, const SpDev *, const int *, long long, const int2 *, const float2 *,
                           const float * );
cudaError_t launch_gather( cudaStream_t, int, int, const SpDev *, const RunDev *, const int *, int, float, float, int, float * );
cudaError_t launch_dep_charge( cudaStream_t, int, int, const SpDev *, const RunDev *, float *, int, int );
cudaError_t launch_phasespace( cudaStream_t, int, int, const SpDev *, const RunDev *, PhaSpec, float * );
cudaError_t launch_energy_sum( cudaStream_t, const SpDev *, int, int, double * );
cudaError_t launch_np_stats( cudaStream_t, const SpDev *, int, unsigned long long * );
cudaError_t launch_reorder( cudaStream_t, const Item *, int, const SpDev *, const RunDev *, int );
cudaError_t launch_current_gc( cudaStream_t, const TileItem *, int, const RunDev *, int );
cudaError_t launch_emf_gc( cudaStream_t, const TileItem *, int, const RunDev *, int, int, int );
cudaError_t launch_cur_gc( cudaStream_t, const TileItem *, int, const RunDev *, int, int );
cudaError_t launch_yee( cudaStream_t, const TileItem *, int, const RunDev *, int, int, int, int, int );
cudaError_t launch_emf_bc( cudaStream_t, const RunDev *, int, int, int );
cudaError_t launch_cur_bc( cudaStream_t, const RunDev *, int, int, int );
cudaError_t launch_kernel3( cudaStream_t, const TileItem *, int, const RunDev *, int, int, float, float, float, int );
cudaError_t launch_shift_left( cudaStream_t, const TileItem *, int, const RunDev *, int );
cudaError_t launch_field_energy( cudaStream_t, const RunDev *, int, int, double * );
cudaError_t launch_grid_add( cudaStream_t, float *, const float *, size_t );
cudaError_t launch_charge_finish( cudaStream_t, const float *, float *, int, int, int, int, int, int, int, int );
cudaError_t launch_grid_gather( cudaStream_t, const float *, float *, int, int, int, int, int, int, int, int );
}  // namespace zb

using namespace zb;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;
static thread_local int g_device = -1;

static int fail( int code, const std::string & msg ) { g_err = msg; return code; }

namespace zb {
// Sets the message zpic_b200_last_error() returns (for entry points in other files).
void set_last_error( const std::string & msg ) { g_err = msg; }
}

#define CK( call )                                                                              \
    do {                                                                                        \
        cudaError_t e_ = ( call );                                                              \
        if ( e_ != cudaSuccess )                                                                \
            return fail( ZPIC_E_CUDA, std::string( #call ) + ": " + cudaGetErrorString( e_ ) ); \
    } while ( 0 )

#define TRY( call ) do { int r_ = ( call ); if ( r_ != ZPIC_OK ) return r_; } while ( 0 )

// Device work of the step paths goes through DEV: when a moving-window step
// is replayed from a CUDA graph, the same host code runs once more for its
// bookkeeping with g_dry set, and issues nothing.
static thread_local bool g_dry = false;
#define DEV( call ) do { if ( !g_dry ) CK( call ); } while ( 0 )

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
struct MovingWindow {          // moving_window.h:1-57
    bool active = false; unsigned n_move = 0; double dx = 0;
    void init( float d ) { active = true; n_move = 0; dx = d; }
    void advance() { if ( active ) n_move++; }
    double motion() const { return n_move * dx; }
    bool needs_move( double t ) const { return active && ( t > dx * ( n_move + 1 ) ); }
};

template < class T > static int dalloc( T ** p, size_t n ) {
    *p = nullptr;
    if ( n == 0 ) n = 1;
    cudaError_t e = cudaMalloc( (void **) p, n * sizeof( T ) );
    if ( e != cudaSuccess ) return fail( ZPIC_E_NOMEM, std::string( "cudaMalloc: " ) + cudaGetErrorString( e ) );
    return ZPIC_OK;
}
template < class T > static void dfree( T *& p ) { if ( p ) cudaFree( p ); p = nullptr; }

static inline int roundup4( int n ) { return ( n + 3 ) & ~3; }
constexpr int MAX_SPECIES = 64;     // species per simulation

enum Phase { PH_PARTICLES = 0, PH_SORT, PH_CURRENT, PH_FIELDS, PH_OTHER, PH_N };

// Steps between in-tile reorders of the particles (option "reorder").  By
// default (-1, automatic) every 50 steps, but never in a moving-window run:
// there the plasma is cold and new particles arrive in injection order every
// step, so the order hardly decays.  On the uniform plasma the particle
// kernel takes 4.56 ms per step right after a reorder and 4.95 ms a hundred
// steps later; a reorder costs ~3.9 ms, 0.08 ms per step at this interval.
constexpr int REORDER_DEFAULT = -1;
constexpr int REORDER_AUTO_STEPS = 50;

// ---------------------------------------------------------------------------
// species
// ---------------------------------------------------------------------------
struct HSpecies {
    std::string name;
    float m_q = -1; uint32_t ppc[2] = { 1, 1 };
    zpic_density dens{}; zpic_udist ud{};
    int push_type = 0;
    int bc[4] = { 1, 1, 1, 1 };
    int id = 0;
    float q = 0, dx[2] = { 0, 0 }, box[2] = { 0, 0 }, dt = 0;
    int iter = 0;
    MovingWindow mw;
    int ntiles = 0;
    uint32_t max_part = 0;
    uint64_t np_bound = 0;    // upper bound of the particle count (capacity checks)
    int grows = 0;            // particle-buffer growths so far
    int pool_h = 0;           // host copy of the pool start at the last upload (copy source)
    SpDev d{};                // descriptor (device pointers)
    bool sort_pending = false;
    bool counters_dirty = false;
    int energy_items = 0;      // per-item energy partials written by the last push
    float * inj_dyn = nullptr;         // window-dependent injection parameters (device)
    unsigned * mw_nmove_d = nullptr;   // device copy of the window's move count

    void free_all() {
        PartArrays * arrs[2] = { &d.A, &d.B };
        for ( auto * a : arrs ) { dfree( a->cell ); dfree( a->xx ); dfree( a->xy ); dfree( a->ux ); dfree( a->uy ); dfree( a->uz ); }
        dfree( d.np ); dfree( d.off ); dfree( d.cap ); dfree( d.nidx ); dfree( d.idx );
        dfree( d.aux ); dfree( d.aux2 ); dfree( d.in_cnt ); dfree( d.stage_cnt );
        dfree( d.cnt ); dfree( d.base ); dfree( d.hs ); dfree( d.overflow ); dfree( d.reloc ); dfree( d.pool );
        dfree( d.rel_tile ); dfree( d.rel_start ); dfree( d.rel_n );
        dfree( d.new_off ); dfree( d.new_cap ); dfree( d.new_np ); dfree( d.extra ); dfree( d.mode );
        dfree( d.energy ); dfree( d.nmove ); dfree( inj_dyn ); dfree( mw_nmove_d );
    }
};

static int alloc_arrays( PartArrays & a, size_t n ) {
    TRY( dalloc( &a.cell, n ) ); TRY( dalloc( &a.xx, n ) ); TRY( dalloc( &a.xy, n ) );
    TRY( dalloc( &a.ux, n ) ); TRY( dalloc( &a.uy, n ) ); TRY( dalloc( &a.uz, n ) );
    return ZPIC_OK;
}

// ---------------------------------------------------------------------------
// plan: device work lists over a set of simulations
// ---------------------------------------------------------------------------
struct zpic_sim;

struct Plan {
    std::vector<zpic_sim *> sims;
    RunDev * runs_d = nullptr;
    SpDev * sps_d = nullptr;
    std::vector<SpDev> sps_h;
    std::vector<int> sp_sim, sp_local;          // plan species -> (sim index, species index)
    Item * k1_items_d[2] = { nullptr, nullptr }; int n_k1[2] = { 0, 0 };   // boris, euler
    Item * sort_items_d = nullptr; int n_sort = 0;
    int * splist_d = nullptr; int n_sp = 0;
    int * rlist_d = nullptr;        // [1 + n_sp] species repacking in the current sort (count, then indices)
    // the same work lists grouped per species (fine-grained species calls)
    Item * spk1_d = nullptr;
    std::vector<int> sp_k1_off, sp_k1_n, sp_sort_off, sp_sort_n;
    TileItem * tile_items_d = nullptr; int n_tiles = 0;
    int max_tile_vol = 0;
    int max_cells = 0, max_guard = 0;   // cells and guard cells of the largest tile
    int max_nxy = 0;                // tile rows (cells in y) of the tallest tile
    int jacc = 0;                   // tile current accumulation (option "jacc")
    int tile_n = 0;                 // n when every run has n x n tiles with a specialised kernel
    int max_tile_cells = 0;         // cells of the largest tile (without guard cells)
    int reorder_every = 0;          // steps between in-tile reorders (option "reorder"; 0: never)
    int reorder_count = 0;          // steps since the last reorder
    bool needs_bc_or_filter = false;
    cudaGraphExec_t graph = nullptr;
    int graph_kernels = 0;
    // in-graph phase timing (profile 2): the captured graph and its event-record
    // nodes, pointed at fresh events before every replay
    struct TimedPhase { int ph; int nl; cudaGraphNode_t na, nb; cudaEvent_t ea, eb; };
    cudaGraph_t graph_src = nullptr;
    std::vector<TimedPhase> timed;
    // moving-window steps, one graph per pattern of window moves
    std::map<unsigned, std::pair<cudaGraphExec_t, int>> mw_graphs;
    bool built = false;

    void drop_step_graph() {
        if ( graph ) { cudaGraphExecDestroy( graph ); graph = nullptr; }
        if ( graph_src ) { cudaGraphDestroy( graph_src ); graph_src = nullptr; }
        for ( auto & t : timed ) { cudaEventDestroy( t.ea ); cudaEventDestroy( t.eb ); }
        timed.clear();
    }
    // a second stream for the field half of a step: after the particle
    // kernel, the tile sort (particle arrays only) and the current and field
    // solve (grids only) are independent and run side by side
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;

    void release() {
        drop_step_graph();
        if ( fork ) { cudaEventDestroy( fork ); fork = nullptr; }
        if ( join ) { cudaEventDestroy( join ); join = nullptr; }
        if ( side ) { cudaStreamDestroy( side ); side = nullptr; }
        for ( auto & g : mw_graphs ) cudaGraphExecDestroy( g.second.first );
        mw_graphs.clear();
        dfree( runs_d ); dfree( sps_d ); dfree( k1_items_d[0] ); dfree( k1_items_d[1] );
        dfree( sort_items_d ); dfree( splist_d ); dfree( rlist_d ); dfree( tile_items_d ); dfree( spk1_d );
        built = false;
    }
};

// ---------------------------------------------------------------------------
// simulation
// ---------------------------------------------------------------------------
struct zpic_sim {
    int device = 0;
    cudaStream_t stream = nullptr;
    int ntx, nty, nxx, nxy;
    float box[2]; double dt;
    float dx[2];
    unsigned iter = 0;
    // EMF (emf.h)
    int emf_bc[4] = { 1, 1, 1, 1 };
    int emf_iter = 0; MovingWindow emf_mw;
    // Current (current.h)
    int cur_bc[4] = { 1, 1, 1, 1 };
    int cur_iter = 0; MovingWindow cur_mw;
    int ftype = 0, fdir = 0; unsigned forder = 1;
    bool j_final = false;          // J holds the summed current, else Jdep holds raw deposits
    bool jdep_clean = true;
    // device
    RunDev run{};
    int * status = nullptr;
    double * dscratch = nullptr;   // small device scratch (energies, stats)
    double * fe_part_d = nullptr;  // per-tile field-energy partials (6 per tile), device
    double * fe_part_h = nullptr;  // and their pinned host copy, allocated on first use
    double * hscratch = nullptr;   // pinned host mirror
    int * shifts_d = nullptr;
    std::vector<HSpecies *> species;
    Plan plan;
    // options
    bool use_graph = true;
    int reorder_every = REORDER_DEFAULT;
    int chunks_opt = 0;
    int jacc = 2;                   // fixed-point tile current (option "jacc")
    double pool_frac = 0.25;        // share of free particle capacity kept as the pool (option "pool_fraction")
    double reloc_room = 0.5;        // room for a relocated tile, share of its count (option "relocation_room")
    // Initial particle capacity per cell and ppc (option "capacity_factor").
    // The reference's max_part = 1.2 cells ppc (species.cpp:1752) serves a
    // packed layout that is rebuilt every step; tile slots need room per
    // tile, and with 1.2 a filamenting Weibel plasma rebuilt its slots every
    // ~15 steps (9.0 k vs 9.3 k run-steps/s on the 256-run ensemble at 1.6).
    double capacity_factor = 1.6;
    int profile = 0;                // 1: per-phase events, steps issued eagerly; 2: the same inside CUDA graphs
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pending[PH_N];
    double phase_ms[PH_N] = { 0 };
    uint64_t phase_launches[PH_N] = { 0 };
    uint64_t launches = 0;
    uint64_t layout_gen = 0;        // bumped when device buffers or descriptors change (batch plans rebuild)

    int tile_vol() const { return run.tile_vol; }
    size_t grid_floats() const { return (size_t) run.tile_vol * ntx * nty * 3; }
};

struct zpic_batch {
    std::vector<zpic_sim *> sims;
    cudaStream_t stream = nullptr;
    Plan plan;
    cudaEvent_t ev = nullptr;
    uint64_t launches = 0;          // kernels launched by batch steps
    int chunks = 0;                 // CTAs per tile chosen for the batch (0 = automatic)
    std::vector<uint64_t> gens;     // layout_gen of each run when the plan was built
};

static int sim_select( zpic_sim * s ) {
    if ( !s ) return fail( ZPIC_E_INVALID, "null simulation handle" );
    CK( cudaSetDevice( s->device ) );
    return ZPIC_OK;
}

// Reads the kernels' status word.  A failure is reported once: the word is
// cleared when it is read, so a later call starts clean (the state the
// failed work left behind is not repaired).
static int check_status( zpic_sim * s ) {
    int st = 0;
    CK( cudaMemcpyAsync( &st, s->status, sizeof( int ), cudaMemcpyDeviceToHost, s->stream ) );
    CK( cudaStreamSynchronize( s->stream ) );
    if ( st & ( ST_WAIT_TIMEOUT | ST_CAPACITY | ST_BAD_CELL ) ) {
        CK( cudaMemsetAsync( s->status, 0, sizeof( int ), s->stream ) );
        CK( cudaStreamSynchronize( s->stream ) );
        std::string m = "device reported:";
        if ( st & ST_WAIT_TIMEOUT ) m += " bounded wait expired;";
        if ( st & ST_CAPACITY ) m += " particle buffer capacity exceeded;";
        if ( st & ST_BAD_CELL ) m += " particle moved more than one tile;";
        return fail( ZPIC_E_DEVICE, m );
    }
    return ZPIC_OK;
}

// Chunks (CTAs) per tile for the particle kernel: enough work items to fill
// the GPU a few times over (the reference splits tiles over blockIdx.z the
// same way, cuda/em2d/species.cpp:924-937).
static int auto_chunks( int ntiles_total, int opt ) {
    if ( opt > 0 ) return opt;
    int dev = 0; cudaGetDevice( &dev );
    int sms = 148; cudaDeviceGetAttribute( &sms, cudaDevAttrMultiProcessorCount, dev );
    const int target = sms * 8;
    if ( ntiles_total >= target ) return 1;
    return std::min( 64, ( target + ntiles_total - 1 ) / ntiles_total );
}

// CTAs per tile of the particle kernel ("chunks" option): n > 0 for every
// tile; 0, the automatic choice, for every tile; -1 balanced: a tile of
// average occupancy gets the automatic number of CTAs, a fuller tile
// proportionally more (up to twice as many), a sparser one fewer, so that
// every CTA moves about the same number of particles however unevenly the
// plasma fills the tiles (faster once a Weibel plasma has filamented, slower
// for uniform plasmas and for runs with many empty tiles).
static void set_chunks( zpic_sim * s ) {
    int ntot = 0; uint64_t np = 0;
    for ( auto * h : s->species ) { ntot += h->ntiles; np += h->np_bound; }
    const int base = auto_chunks( std::max( 1, ntot ), std::max( 0, s->chunks_opt ) );
    for ( auto * h : s->species ) {
        if ( s->chunks_opt >= 0 ) { h->d.nchunk = base; h->d.chunk_target = 0; continue; }
        h->d.nchunk = std::min( 64, 2 * base );
        const uint64_t per_tile = ( np + ntot - 1 ) / std::max( 1, ntot );
        h->d.chunk_target = (int) std::max<uint64_t>( 256, ( per_tile + base - 1 ) / base );
    }
}

static int upload_run( zpic_sim * s ) {
    RunDev & R = s->run;
    R.emf_perx = s->emf_bc[0] == ZPIC_EMF_BC_PERIODIC; R.emf_pery = s->emf_bc[2] == ZPIC_EMF_BC_PERIODIC;
    R.cur_perx = s->cur_bc[0] == ZPIC_CURRENT_BC_PERIODIC; R.cur_pery = s->cur_bc[2] == ZPIC_CURRENT_BC_PERIODIC;
    for ( int k = 0; k < 4; k++ ) { R.emf_bc[k] = s->emf_bc[k]; R.cur_bc[k] = s->cur_bc[k]; }
    s->plan.built = false;
    s->layout_gen++;
    return ZPIC_OK;
}

// Build the work lists for a set of simulations (one sim, or a batch).
static int plan_build( Plan & P, const std::vector<zpic_sim *> & sims, int chunks_override = 0 ) {
    P.release();
    P.sims = sims;
    std::vector<RunDev> runs;
    std::vector<Item> k1[2], sort_items, spk1;
    std::vector<int> splist;
    std::vector<TileItem> tiles;
    P.sps_h.clear(); P.sp_sim.clear(); P.sp_local.clear();
    P.sp_k1_off.clear(); P.sp_k1_n.clear(); P.sp_sort_off.clear(); P.sp_sort_n.clear();
    P.max_tile_vol = 0;
    P.max_cells = 0; P.max_guard = 0; P.max_tile_cells = 0; P.max_nxy = 0;
    P.reorder_every = 0; P.reorder_count = 0;
    P.jacc = -1;
    P.tile_n = -1;
    P.needs_bc_or_filter = false;
    int total_tiles = 0;
    for ( auto * s : sims ) for ( auto * sp : s->species ) { (void) sp; total_tiles += s->ntx * s->nty; }
    // a batch chooses its CTAs per tile from all of its tiles; a single
    // simulation keeps the choice made for it
    const int batch_chunks = chunks_override > 0 ? chunks_override
                           : sims.size() > 1 ? auto_chunks( std::max( 1, total_tiles ), 0 ) : 0;
    for ( size_t r = 0; r < sims.size(); r++ ) {
        zpic_sim * s = sims[r];
        runs.push_back( s->run );
        P.max_tile_vol = std::max( P.max_tile_vol, s->run.tile_vol );
        P.max_cells = std::max( P.max_cells, s->run.extx * s->run.exty );
        P.max_guard = std::max( P.max_guard, s->run.extx * s->run.exty - s->run.nxx * s->run.nxy );
        P.max_tile_cells = std::max( P.max_tile_cells, s->run.nxx * s->run.nxy );
        P.max_nxy = std::max( P.max_nxy, s->run.nxy );
        // a batch reorders as often as its most frequent run asks
        const int every = s->reorder_every >= 0 ? s->reorder_every : ( s->emf_mw.active ? 0 : REORDER_AUTO_STEPS );
        if ( every > 0 )
            P.reorder_every = P.reorder_every > 0 ? std::min( P.reorder_every, every ) : every;
        // one accumulation mode per plan: the runs' own when they agree
        P.jacc = ( P.jacc < 0 || P.jacc == s->jacc ) ? s->jacc : 2;
        const int tn = ( s->nxx == 16 && s->nxy == 16 ) ? 16 : 0;
        P.tile_n = ( P.tile_n < 0 || P.tile_n == tn ) ? tn : 0;
        for ( int t = 0; t < s->ntx * s->nty; t++ ) tiles.push_back( { (int) r, t } );
        for ( int k = 0; k < 4; k++ )
            if ( s->emf_bc[k] > ZPIC_EMF_BC_PERIODIC || s->cur_bc[k] > ZPIC_CURRENT_BC_PERIODIC ) P.needs_bc_or_filter = true;
        if ( s->ftype != ZPIC_FILTER_NONE || s->emf_mw.active ) P.needs_bc_or_filter = true;
    }
    for ( size_t r = 0; r < sims.size(); r++ ) {
        zpic_sim * s = sims[r];
        for ( size_t k = 0; k < s->species.size(); k++ ) {
            HSpecies * sp = s->species[k];
            SpDev d = sp->d;
            if ( batch_chunks ) { d.nchunk = batch_chunks; d.chunk_target = 0; }
            d.run = (int) r;
            const int gi = (int) P.sps_h.size();
            P.sps_h.push_back( d );
            P.sp_sim.push_back( (int) r ); P.sp_local.push_back( (int) k );
            splist.push_back( gi );
            P.sp_k1_off.push_back( (int) spk1.size() );
            P.sp_sort_off.push_back( (int) sort_items.size() );
            for ( int t = 0; t < sp->ntiles; t++ ) {
                for ( int c = 0; c < d.nchunk; c++ ) {
                    k1[ sp->push_type ? 1 : 0 ].push_back( { gi, t, c, 0 } );
                    spk1.push_back( { gi, t, c, 0 } );
                }
                sort_items.push_back( { gi, t, 0, 0 } );
            }
            P.sp_k1_n.push_back( (int) spk1.size() - P.sp_k1_off.back() );
            P.sp_sort_n.push_back( (int) sort_items.size() - P.sp_sort_off.back() );
        }
    }
    P.n_sp = (int) splist.size();
    TRY( dalloc( &P.runs_d, runs.size() ) );
    TRY( dalloc( &P.sps_d, P.sps_h.size() ) );
    TRY( dalloc( &P.splist_d, splist.size() ) );
    TRY( dalloc( &P.rlist_d, splist.size() + 1 ) );
    CK( cudaMemset( P.rlist_d, 0, ( splist.size() + 1 ) * sizeof( int ) ) );
    TRY( dalloc( &P.tile_items_d, tiles.size() ) );
    TRY( dalloc( &P.sort_items_d, sort_items.size() ) );
    CK( cudaStreamCreateWithFlags( &P.side, cudaStreamNonBlocking ) );
    CK( cudaEventCreateWithFlags( &P.fork, cudaEventDisableTiming ) );
    CK( cudaEventCreateWithFlags( &P.join, cudaEventDisableTiming ) );
    CK( cudaMemcpy( P.runs_d, runs.data(), runs.size() * sizeof( RunDev ), cudaMemcpyHostToDevice ) );
    if ( !P.sps_h.empty() ) {
        CK( cudaMemcpy( P.sps_d, P.sps_h.data(), P.sps_h.size() * sizeof( SpDev ), cudaMemcpyHostToDevice ) );
        CK( cudaMemcpy( P.splist_d, splist.data(), splist.size() * sizeof( int ), cudaMemcpyHostToDevice ) );
        CK( cudaMemcpy( P.sort_items_d, sort_items.data(), sort_items.size() * sizeof( Item ), cudaMemcpyHostToDevice ) );
    }
    CK( cudaMemcpy( P.tile_items_d, tiles.data(), tiles.size() * sizeof( TileItem ), cudaMemcpyHostToDevice ) );
    for ( int p = 0; p < 2; p++ ) {
        P.n_k1[p] = (int) k1[p].size();
        TRY( dalloc( &P.k1_items_d[p], k1[p].size() ) );
        if ( !k1[p].empty() )
            CK( cudaMemcpy( P.k1_items_d[p], k1[p].data(), k1[p].size() * sizeof( Item ), cudaMemcpyHostToDevice ) );
    }
    TRY( dalloc( &P.spk1_d, spk1.size() ) );
    if ( !spk1.empty() )
        CK( cudaMemcpy( P.spk1_d, spk1.data(), spk1.size() * sizeof( Item ), cudaMemcpyHostToDevice ) );
    P.n_sort = (int) sort_items.size();
    P.n_tiles = (int) tiles.size();
    P.built = true;
    return ZPIC_OK;
}

// ---------------------------------------------------------------------------
// profiling helpers
// ---------------------------------------------------------------------------
// Phase events recorded while a step graph is captured for in-graph timing
// (profile 2): they become event-record nodes, listed here with their phase.
struct CapturedPhase { int ph; int nl; cudaEvent_t a, b; };
static thread_local bool g_capture_timing = false;
static thread_local std::vector<CapturedPhase> g_cap_events;

// Inside a step graph only the particle phase is timed (two event nodes per
// step: the nodes serialise with the kernels around them and cost about 1 us
// each).
struct PhaseScope {
    zpic_sim * s; cudaStream_t st; int ph; cudaEvent_t a = nullptr, b = nullptr; int nl; bool on = false;
    PhaseScope( zpic_sim * s_, cudaStream_t st_, int ph_, int nlaunch ) : s( s_ ), st( st_ ), ph( ph_ ), nl( nlaunch ) {
        on = s && s->profile && ( !g_capture_timing || ph == PH_PARTICLES );
        if ( on ) {
            cudaEventCreate( &a ); cudaEventCreate( &b );
            if ( g_capture_timing ) cudaEventRecordWithFlags( a, st, cudaEventRecordExternal );
            else cudaEventRecord( a, st );
        }
    }
    ~PhaseScope() {
        if ( !s ) return;
        s->launches += nl;
        s->phase_launches[ph] += nl;
        if ( on ) {
            if ( g_capture_timing ) {
                cudaEventRecordWithFlags( b, st, cudaEventRecordExternal );
                g_cap_events.push_back( { ph, nl, a, b } );
            } else {
                cudaEventRecord( b, st );
                s->ev_pending[ph].push_back( { a, b } );
            }
        }
    }
};

static void resolve_phase_events( zpic_sim * s ) {
    for ( int p = 0; p < PH_N; p++ ) {
        for ( auto & e : s->ev_pending[p] ) {
            float ms = 0;
            cudaEventSynchronize( e.second );
            cudaEventElapsedTime( &ms, e.first, e.second );
            s->phase_ms[p] += ms;
            cudaEventDestroy( e.first ); cudaEventDestroy( e.second );
        }
        s->ev_pending[p].clear();
    }
}

// ---------------------------------------------------------------------------
// step pieces
// ---------------------------------------------------------------------------
static zpic_sim * prof_sim( Plan & P ) { return P.sims.size() == 1 ? P.sims[0] : nullptr; }

// push + move + deposit + walls + leaver detection for all species of the plan
static int run_particles( Plan & P, cudaStream_t st, int push, int move, const int * shifts ) {
    for ( int p = 0; p < 2; p++ ) {
        if ( P.n_k1[p] == 0 ) continue;
        PhaseScope ps( prof_sim( P ), st, PH_PARTICLES, 1 );
        DEV( launch_particles( st, push ? p + 1 : 0, move, 1, P.k1_items_d[p], P.n_k1[p], P.sps_d, P.runs_d, shifts, P.max_tile_vol,
                              P.jacc, P.tile_n ) );
    }
    return ZPIC_OK;
}

static int run_sort( Plan & P, cudaStream_t st, int use_extra ) {
    if ( P.n_sp == 0 ) return ZPIC_OK;
    PhaseScope ps( prof_sim( P ), st, PH_SORT, 4 );
    DEV( launch_sort( st, P.sort_items_d, P.n_sort, P.sps_d, P.splist_d, P.n_sp, P.runs_d, use_extra, P.rlist_d ) );
    return ZPIC_OK;
}

// Current::advance device part for every run of the plan (current.cpp:227-246)
static int run_current( Plan & P, cudaStream_t st ) {
    {
        PhaseScope ps( prof_sim( P ), st, PH_CURRENT, 1 );
        DEV( launch_current_gc( st, P.tile_items_d, P.n_tiles, P.runs_d, P.max_cells ) );
    }
    if ( !P.needs_bc_or_filter ) return ZPIC_OK;
    for ( size_t r = 0; r < P.sims.size(); r++ ) {
        zpic_sim * s = P.sims[r];
        if ( s->cur_bc[0] > 1 || s->cur_bc[1] > 1 ) {
            PhaseScope ps( prof_sim( P ), st, PH_CURRENT, 1 );
            DEV( launch_cur_bc( st, P.runs_d, (int) r, 0, 2 * s->nty * s->run.exty ) );
        }
        if ( s->cur_bc[2] > 1 || s->cur_bc[3] > 1 ) {
            PhaseScope ps( prof_sim( P ), st, PH_CURRENT, 1 );
            DEV( launch_cur_bc( st, P.runs_d, (int) r, 1, 2 * s->ntx * s->run.extx ) );
        }
    }
    // filters (filter.h:22-86): run-specific, launched over all tiles of the plan only when uniform
    for ( size_t r = 0; r < P.sims.size(); r++ ) {
        zpic_sim * s = P.sims[r];
        if ( s->ftype == ZPIC_FILTER_NONE ) continue;
        const unsigned order = s->forder > 0 ? s->forder : 1;
        // tile items of this run only
        int first = 0;
        for ( size_t q = 0; q < r; q++ ) first += P.sims[q]->ntx * P.sims[q]->nty;
        const int nt = s->ntx * s->nty;
        const TileItem * items = P.tile_items_d + first;
        auto pass = [&]( float a, float b, float c ) -> int {
            PhaseScope ps( prof_sim( P ), st, PH_CURRENT, 2 );
            DEV( launch_kernel3( st, items, nt, P.runs_d, 2, s->fdir, a, b, c, P.max_tile_vol ) );
            DEV( launch_cur_gc( st, items, nt, P.runs_d, s->fdir ? 2 : 1, P.max_guard ) );
            return ZPIC_OK;
        };
        for ( unsigned i = 0; i < order; i++ ) TRY( pass( 0.25f, 0.5f, 0.25f ) );
        if ( s->ftype == ZPIC_FILTER_COMPENSATED ) {
            const float a = -1.0f;
            const float b = ( 4.0 + 2.0 * order ) / order;
            const float norm = 2 * a + b;
            TRY( pass( a / norm, b / norm, a / norm ) );
        }
    }
    return ZPIC_OK;
}

// EMF::advance device part (emf.cpp:513-580 and 135-194): Yee, guard cells, bc.
// with_shift: EMF::move_window (emf.cpp:120-129) follows at once in a run
// without physical boundaries; the Yee kernel writes its tiles shifted and
// the guard refresh completes the shift (two kernels instead of four).
static int run_fields( Plan & P, cudaStream_t st, int with_j, int j_raw, int clear_jdep, bool with_shift = false ) {
    if ( with_shift ) {
        PhaseScope ps( prof_sim( P ), st, PH_FIELDS, 2 );
        DEV( launch_yee( st, P.tile_items_d, P.n_tiles, P.runs_d, with_j, j_raw, clear_jdep, P.max_tile_vol, 1 ) );
        DEV( launch_emf_gc( st, P.tile_items_d, P.n_tiles, P.runs_d, 3, P.max_guard, P.max_nxy ) );
        return ZPIC_OK;
    }
    {
        PhaseScope ps( prof_sim( P ), st, PH_FIELDS, 2 );
        DEV( launch_yee( st, P.tile_items_d, P.n_tiles, P.runs_d, with_j, j_raw, clear_jdep, P.max_tile_vol, 0 ) );
        DEV( launch_emf_gc( st, P.tile_items_d, P.n_tiles, P.runs_d, 3, P.max_guard, 0 ) );
    }
    if ( !P.needs_bc_or_filter ) return ZPIC_OK;
    for ( size_t r = 0; r < P.sims.size(); r++ ) {
        zpic_sim * s = P.sims[r];
        if ( s->emf_bc[0] > 1 || s->emf_bc[1] > 1 ) {
            PhaseScope ps( prof_sim( P ), st, PH_FIELDS, 1 );
            DEV( launch_emf_bc( st, P.runs_d, (int) r, 0, 2 * s->nty * s->run.exty ) );
        }
        if ( s->emf_bc[2] > 1 || s->emf_bc[3] > 1 ) {
            PhaseScope ps( prof_sim( P ), st, PH_FIELDS, 1 );
            DEV( launch_emf_bc( st, P.runs_d, (int) r, 1, 2 * s->ntx * s->run.extx ) );
        }
    }
    return ZPIC_OK;
}

// EMF::move_window (emf.cpp:120-129) for one run of the plan
static int run_shift( Plan & P, cudaStream_t st, int r ) {
    int first = 0;
    for ( int q = 0; q < r; q++ ) first += P.sims[q]->ntx * P.sims[q]->nty;
    const int nt = P.sims[r]->ntx * P.sims[r]->nty;
    PhaseScope ps( prof_sim( P ), st, PH_FIELDS, 2 );
    DEV( launch_shift_left( st, P.tile_items_d + first, nt, P.runs_d, P.max_tile_vol ) );
    DEV( launch_emf_gc( st, P.tile_items_d + first, nt, P.runs_d, 1, P.max_guard, 0 ) );
    return ZPIC_OK;
}

static int ensure_plan( zpic_sim * s ) {
    if ( !s->plan.built ) TRY( plan_build( s->plan, { s } ) );
    return ZPIC_OK;
}

static int ensure_jdep_clean( zpic_sim * s, cudaStream_t st ) {
    if ( !s->jdep_clean ) {
        DEV( cudaMemsetAsync( s->run.Jdep, 0, s->grid_floats() * sizeof( float ), st ) );
        s->jdep_clean = true;
    }
    return ZPIC_OK;
}

// One Simulation::advance (simulation.h:90-107) for all sims of a plan, on st.
static int plan_step_device( Plan & P, cudaStream_t st ) {
    TRY( run_particles( P, st, 1, 2, nullptr ) );
    // the sort on the simulation's stream, current and fields on the side
    // stream (forked after the particle kernel, joined before the step ends)
    DEV( cudaEventRecord( P.fork, st ) );
    DEV( cudaStreamWaitEvent( P.side, P.fork, 0 ) );
    TRY( run_current( P, P.side ) );
    TRY( run_fields( P, P.side, 1, 0, 1 ) );
    DEV( cudaEventRecord( P.join, P.side ) );
    TRY( run_sort( P, st, 0 ) );
    DEV( cudaStreamWaitEvent( st, P.join, 0 ) );
    return ZPIC_OK;
}

static void plan_step_host( Plan & P ) {
    for ( size_t g = 0; g < P.sps_h.size(); g++ )
        P.sims[ P.sp_sim[g] ]->species[ P.sp_local[g] ]->energy_items = P.sps_h[g].ntiles * P.sps_h[g].nchunk;
    for ( auto * s : P.sims ) {
        for ( auto * sp : s->species ) { sp->iter++; sp->sort_pending = false; sp->counters_dirty = false; }
        s->cur_iter++;
        if ( s->cur_mw.needs_move( s->cur_iter * s->dt ) ) s->cur_mw.advance();
        s->emf_iter++;
        s->j_final = true;
        s->jdep_clean = true;
        s->iter++;
    }
}

static int count_graph_kernels( cudaGraph_t g ) {
    size_t n = 0;
    cudaGraphGetNodes( g, nullptr, &n );
    std::vector<cudaGraphNode_t> nodes( n );
    cudaGraphGetNodes( g, nodes.data(), &n );
    int k = 0;
    for ( auto & nd : nodes ) { cudaGraphNodeType t; cudaGraphNodeGetType( nd, &t ); if ( t == cudaGraphNodeTypeKernel ) k++; }
    return k;
}

// In-tile reorder of every species after a complete step, every
// reorder_every steps (the particles' order only; no physics changes).
static int maybe_reorder( Plan & P, cudaStream_t st, uint64_t * launches ) {
    if ( P.reorder_every <= 0 || ++P.reorder_count < P.reorder_every ) return ZPIC_OK;
    P.reorder_count = 0;
    PhaseScope ps( prof_sim( P ), st, PH_OTHER, 0 );
    CK( launch_reorder( st, P.sort_items_d, P.n_sort, P.sps_d, P.runs_d, P.max_tile_cells ) );
    if ( launches ) *launches += 1;
    return ZPIC_OK;
}

static int plan_advance( Plan & P, cudaStream_t st, int nsteps, bool use_graph, uint64_t * launches ) {
    for ( auto * s : P.sims ) TRY( ensure_jdep_clean( s, st ) );
    const bool can_graph = use_graph && nsteps > 1;
    zpic_sim * ts = prof_sim( P );
    const bool timing = ts && ts->profile == 2;
    if ( can_graph && P.graph && timing != !P.timed.empty() ) P.drop_step_graph();
    if ( can_graph && !P.graph ) {
        // Capture one step.  Launch counting is suspended during capture
        // (replays count the graph's kernel nodes instead), and so is
        // profiling unless the phases are to be timed inside the graph.
        std::vector<uint64_t> l0;
        std::vector<int> prof;
        uint64_t pl0[PH_N] = { 0 };
        if ( timing ) for ( int p = 0; p < PH_N; p++ ) pl0[p] = ts->phase_launches[p];
        for ( auto * s : P.sims ) {
            l0.push_back( s->launches ); prof.push_back( s->profile );
            if ( !timing ) s->profile = 0;
        }
        g_capture_timing = timing;
        g_cap_events.clear();
        cudaGraph_t g;
        CK( cudaStreamBeginCapture( st, cudaStreamCaptureModeThreadLocal ) );
        const int rc = plan_step_device( P, st );
        const cudaError_t e = cudaStreamEndCapture( st, &g );
        g_capture_timing = false;
        for ( size_t i = 0; i < P.sims.size(); i++ ) { P.sims[i]->launches = l0[i]; P.sims[i]->profile = prof[i]; }
        if ( timing ) for ( int p = 0; p < PH_N; p++ ) ts->phase_launches[p] = pl0[p];
        std::vector<CapturedPhase> cap;
        cap.swap( g_cap_events );
        if ( rc != ZPIC_OK || e != cudaSuccess ) {
            for ( auto & c : cap ) { cudaEventDestroy( c.a ); cudaEventDestroy( c.b ); }
            if ( rc != ZPIC_OK ) return rc;
            return fail( ZPIC_E_CUDA, std::string( "graph capture: " ) + cudaGetErrorString( e ) );
        }
        P.graph_kernels = count_graph_kernels( g );
        if ( timing ) {
            // event-record node of each captured phase event
            size_t n = 0;
            cudaGraphGetNodes( g, nullptr, &n );
            std::vector<cudaGraphNode_t> nodes( n );
            cudaGraphGetNodes( g, nodes.data(), &n );
            std::map<cudaEvent_t, cudaGraphNode_t> node_of;
            for ( auto & nd : nodes ) {
                cudaGraphNodeType t;
                cudaGraphNodeGetType( nd, &t );
                cudaEvent_t ev;
                if ( t == cudaGraphNodeTypeEventRecord && cudaGraphEventRecordNodeGetEvent( nd, &ev ) == cudaSuccess )
                    node_of[ev] = nd;
            }
            for ( auto & c : cap ) {
                auto ia = node_of.find( c.a ), ib = node_of.find( c.b );
                if ( ia != node_of.end() && ib != node_of.end() )
                    P.timed.push_back( { c.ph, c.nl, ia->second, ib->second, c.a, c.b } );
                else { cudaEventDestroy( c.a ); cudaEventDestroy( c.b ); }
            }
        }
        const cudaError_t e2 = cudaGraphInstantiate( &P.graph, g, 0 );
        if ( timing ) P.graph_src = g;
        else cudaGraphDestroy( g );
        if ( e2 != cudaSuccess ) { P.graph = nullptr; P.drop_step_graph(); return fail( ZPIC_E_CUDA, std::string( "graph instantiate: " ) + cudaGetErrorString( e2 ) ); }
    }
    for ( int n = 0; n < nsteps; n++ ) {
        if ( can_graph && P.graph ) {
            if ( timing ) {
                // fresh events for this replay's phase nodes
                for ( auto & t : P.timed ) {
                    cudaEvent_t a, b;
                    CK( cudaEventCreate( &a ) );
                    CK( cudaEventCreate( &b ) );
                    CK( cudaGraphExecEventRecordNodeSetEvent( P.graph, t.na, a ) );
                    CK( cudaGraphExecEventRecordNodeSetEvent( P.graph, t.nb, b ) );
                    ts->ev_pending[t.ph].push_back( { a, b } );
                    ts->phase_launches[t.ph] += t.nl;
                }
            }
            CK( cudaGraphLaunch( P.graph, st ) );
            if ( launches ) *launches += P.graph_kernels;
        } else {
            TRY( plan_step_device( P, st ) );
        }
        plan_step_host( P );
        TRY( maybe_reorder( P, st, launches ) );
    }
    if ( timing && P.graph ) {
        // point the phase nodes back at the capture's own events, so that the
        // replays' events can be destroyed once they have been read
        for ( auto & t : P.timed ) {
            CK( cudaGraphExecEventRecordNodeSetEvent( P.graph, t.na, t.ea ) );
            CK( cudaGraphExecEventRecordNodeSetEvent( P.graph, t.nb, t.eb ) );
        }
    }
    return ZPIC_OK;
}

// ---------------------------------------------------------------------------
// species set-up
// ---------------------------------------------------------------------------

// Slot layout: need[t] = roundup4(np[t]); the free capacity spread over the
// slots in proportion to need + min_slack (multiples of 4), but for a share
// pool_frac left after the last slot as the pool that tiles outgrowing their
// slots move into (the sort's relocation).
static void slot_layout( const std::vector<int> & np, uint64_t max_part, int min_slack, double pool_frac,
                         std::vector<int> & off, std::vector<int> & cap ) {
    const int nt = (int) np.size();
    off.assign( nt, 0 ); cap.assign( nt, 0 );
    long long need_sum = 0, w_sum = 0;
    for ( int t = 0; t < nt; t++ ) { const int nd = roundup4( np[t] ); need_sum += nd; w_sum += nd + min_slack; }
    const long long free_cap = (long long) ( std::max<long long>( 0, (long long) max_part - need_sum ) * ( 1.0 - pool_frac ) );
    long long o = 0;
    for ( int t = 0; t < nt; t++ ) {
        const int nd = roundup4( np[t] );
        const long long sl = w_sum > 0 ? ( free_cap * ( nd + min_slack ) ) / w_sum : 0;
        cap[t] = nd + (int) ( sl & ~3LL );
        off[t] = (int) o;
        o += cap[t];
    }
}

// Upload packed particles (reference layout) into the slot layout of sp.
static int species_upload( zpic_sim * s, HSpecies * sp, const std::vector<int> & np,
                           const int32_t * ix, const float * x, const float * u ) {
    const int nt = sp->ntiles;
    std::vector<int> poff( nt ); long long total = 0;
    for ( int t = 0; t < nt; t++ ) { poff[t] = (int) total; total += np[t]; }
    std::vector<int> off, cap;
    const int min_slack = std::max<int>( 16, (int) ( sp->ppc[0] * sp->ppc[1] * s->nxx * s->nxy / 8 ) );
    slot_layout( np, sp->max_part, min_slack, sp->d.pool_frac, off, cap );
    if ( (long long) off.back() + cap.back() > (long long) sp->max_part || [&] {
             for ( int t = 0; t < nt; t++ ) if ( cap[t] < np[t] ) return true; return false; }() )
        return fail( ZPIC_E_NOMEM, "particle set does not fit the species buffer" );
    cudaStream_t st = s->stream;
    CK( cudaMemcpyAsync( sp->d.np, np.data(), nt * sizeof( int ), cudaMemcpyHostToDevice, st ) );
    CK( cudaMemcpyAsync( sp->d.off, off.data(), nt * sizeof( int ), cudaMemcpyHostToDevice, st ) );
    CK( cudaMemcpyAsync( sp->d.cap, cap.data(), nt * sizeof( int ), cudaMemcpyHostToDevice, st ) );
    sp->pool_h = off.back() + cap.back();
    CK( cudaMemcpyAsync( sp->d.pool, &sp->pool_h, sizeof( int ), cudaMemcpyHostToDevice, st ) );
    int * poff_d = nullptr;
    TRY( dalloc( &poff_d, nt ) );
    CK( cudaMemcpyAsync( poff_d, poff.data(), nt * sizeof( int ), cudaMemcpyHostToDevice, st ) );
    // the species descriptor must be on the device for the unpack kernel
    SpDev * one = nullptr;
    TRY( dalloc( &one, 1 ) );
    CK( cudaMemcpyAsync( one, &sp->d, sizeof( SpDev ), cudaMemcpyHostToDevice, st ) );
    // Chunks of whole tiles staged in buffer B (free outside a step), two in
    // flight: the host-to-device copies of one chunk, on a copy stream,
    // overlap the unpack of the one before.  Even chunks use (B.cell, B.xx,
    // B.ux), odd ones (B.xy, B.uy, B.uz); each array holds max_part 4-byte
    // words, so a chunk holds up to max_part / 3 particles (12 bytes of
    // momentum each).  A tile larger than that is staged in its own buffers.
    const long long chunk_cap = std::max<long long>( 1, (long long) sp->max_part / 3 );
    std::vector<int> cut( 1, 0 );
    bool big = false;
    {
        long long acc = 0;
        for ( int t = 0; t < nt; t++ ) {
            if ( np[t] > chunk_cap ) big = true;
            if ( acc + np[t] > chunk_cap && t > cut.back() ) { cut.push_back( t ); acc = 0; }
            acc += np[t];
        }
        cut.push_back( nt );
    }
    std::vector<int2 *> own_ix; std::vector<float2 *> own_x; std::vector<float *> own_u;
    cudaStream_t cs = nullptr;
    cudaEvent_t copied[2] = { nullptr, nullptr }, unpacked[2] = { nullptr, nullptr };
    CK( cudaStreamCreateWithFlags( &cs, cudaStreamNonBlocking ) );
    for ( int b = 0; b < 2; b++ ) {
        CK( cudaEventCreateWithFlags( &copied[b], cudaEventDisableTiming ) );
        CK( cudaEventCreateWithFlags( &unpacked[b], cudaEventDisableTiming ) );
    }
    // the copy stream starts after the work already on the simulation's stream
    CK( cudaEventRecord( unpacked[0], st ) );
    CK( cudaStreamWaitEvent( cs, unpacked[0], 0 ) );
    int rc = ZPIC_OK;
    for ( size_t k = 0; k + 1 < cut.size() && rc == ZPIC_OK; k++ ) {
        const int t0 = cut[k], t1 = cut[k + 1], b = (int) ( k & 1 );
        const long long p0 = poff[t0], n = ( t1 < nt ? (long long) poff[t1] : total ) - p0;
        int2 * ix_d; float2 * x_d; float * u_d;
        if ( big ) {
            int2 * a = nullptr; float2 * c = nullptr; float * e = nullptr;
            if ( ( rc = dalloc( &a, n ) ) != ZPIC_OK || ( rc = dalloc( &c, n ) ) != ZPIC_OK || ( rc = dalloc( &e, 3 * n ) ) != ZPIC_OK ) {
                dfree( a ); dfree( c ); dfree( e );
                break;
            }
            own_ix.push_back( a ); own_x.push_back( c ); own_u.push_back( e );
            ix_d = a; x_d = c; u_d = e;
        } else {
            ix_d = reinterpret_cast<int2 *>( b ? (void *) sp->d.B.xy : (void *) sp->d.B.cell );
            x_d = reinterpret_cast<float2 *>( b ? sp->d.B.uy : sp->d.B.xx );
            u_d = b ? sp->d.B.uz : sp->d.B.ux;
            if ( k >= 2 ) CK( cudaStreamWaitEvent( cs, unpacked[b], 0 ) );
        }
        if ( n > 0 ) {
            CK( cudaMemcpyAsync( ix_d, ix + 2 * p0, n * sizeof( int2 ), cudaMemcpyHostToDevice, cs ) );
            CK( cudaMemcpyAsync( x_d, x + 2 * p0, n * sizeof( float2 ), cudaMemcpyHostToDevice, cs ) );
            CK( cudaMemcpyAsync( u_d, u + 3 * p0, n * 3 * sizeof( float ), cudaMemcpyHostToDevice, cs ) );
        }
        CK( cudaEventRecord( copied[b], cs ) );
        CK( cudaStreamWaitEvent( st, copied[b], 0 ) );
        CK( launch_unpack( st, 0, t0, t1 - t0, one, poff_d, p0, ix_d, x_d, u_d ) );
        s->launches++;
        CK( cudaEventRecord( unpacked[b], st ) );
    }
    CK( cudaStreamSynchronize( st ) );
    for ( int b = 0; b < 2; b++ ) { cudaEventDestroy( copied[b] ); cudaEventDestroy( unpacked[b] ); }
    cudaStreamDestroy( cs );
    for ( size_t i = 0; i < own_ix.size(); i++ ) { dfree( own_ix[i] ); dfree( own_x[i] ); dfree( own_u[i] ); }
    if ( rc != ZPIC_OK ) { dfree( one ); dfree( poff_d ); return rc; }
    CK( cudaMemsetAsync( sp->d.cnt, 0, 9 * (size_t) nt * sizeof( int ), st ) );
    CK( cudaMemsetAsync( sp->d.nidx, 0, nt * sizeof( int ), st ) );
    CK( cudaStreamSynchronize( st ) );
    dfree( one ); dfree( poff_d );
    sp->np_bound = total;
    sp->sort_pending = false;
    sp->counters_dirty = false;
    return ZPIC_OK;
}

static int species_alloc( zpic_sim * s, HSpecies * sp, uint64_t max_part ) {
    const int nt = s->ntx * s->nty;
    sp->ntiles = nt;
    sp->max_part = (uint32_t) max_part;
    SpDev & d = sp->d;
    d.ntiles = nt;
    d.max_part = (int) max_part;
    TRY( alloc_arrays( d.A, max_part ) );
    TRY( alloc_arrays( d.B, max_part ) );
    TRY( dalloc( &d.np, nt ) ); TRY( dalloc( &d.off, nt ) ); TRY( dalloc( &d.cap, nt ) );
    TRY( dalloc( &d.nidx, nt ) );
    TRY( dalloc( &d.idx, max_part ) ); TRY( dalloc( &d.aux, max_part ) ); TRY( dalloc( &d.aux2, max_part ) );
    TRY( dalloc( &d.in_cnt, nt ) ); TRY( dalloc( &d.stage_cnt, nt ) );
    TRY( dalloc( &d.cnt, 9 * (size_t) nt ) ); TRY( dalloc( &d.base, 9 * (size_t) nt ) );
    TRY( dalloc( &d.hs, nt ) ); TRY( dalloc( &d.overflow, 1 ) );
    TRY( dalloc( &d.reloc, nt ) ); TRY( dalloc( &d.pool, 1 ) );
    TRY( dalloc( &d.rel_tile, nt ) ); TRY( dalloc( &d.rel_start, nt + 1 ) ); TRY( dalloc( &d.rel_n, 1 ) );
    CK( cudaMemset( d.rel_n, 0, sizeof( int ) ) );
    CK( cudaMemset( d.reloc, 0, nt * sizeof( int ) ) );
    CK( cudaMemset( d.pool, 0, sizeof( int ) ) );
    CK( cudaMemset( d.cnt, 0, 9 * (size_t) nt * sizeof( int ) ) );
    CK( cudaMemset( d.overflow, 0, sizeof( int ) ) );
    TRY( dalloc( &d.new_off, nt ) ); TRY( dalloc( &d.new_cap, nt ) ); TRY( dalloc( &d.new_np, nt ) );
    TRY( dalloc( &d.extra, nt ) ); TRY( dalloc( &d.mode, 1 ) );
    TRY( dalloc( &sp->inj_dyn, 4 ) ); TRY( dalloc( &sp->mw_nmove_d, 1 ) );
    CK( cudaMemset( sp->mw_nmove_d, 0, sizeof( unsigned ) ) );
    TRY( dalloc( &d.nmove, 3 ) );
    CK( cudaMemset( d.nmove, 0, 3 * sizeof( unsigned long long ) ) );
    CK( cudaMemset( d.extra, 0, nt * sizeof( int ) ) );
    CK( cudaMemset( d.mode, 0, sizeof( int ) ) );
    return ZPIC_OK;
}

// Capacity a species needs for `total` particles: after a sort every tile's
// slot is rounded up to 4 particles, so up to 3 more per tile.
static uint64_t capacity_for( const HSpecies * h, uint64_t total ) { return total + 4ull * h->ntiles; }

// Particle-buffer growth (Particles::grow_buffer, particles.h:174-190: the
// reference grows its buffers in multiples of 64 Ki particles when a sort's
// new total exceeds max_part, particles.cpp:863-888).  New arrays of new_max
// particles; the live contents are copied -- the tile slots of A, and the
// leaver outbox (B) and leaver lists (idx) that a pending sort still reads --
// the new room lies after the last slot (the next repack spreads it over the
// tiles).  The plans' device copies of the descriptor are rewritten in
// place, so that step graphs already captured (their kernels read the
// descriptor from device memory) run on the new buffers.
static int species_grow( zpic_sim * s, HSpecies * h, uint64_t new_max ) {
    new_max = ( new_max + 65535 ) & ~(uint64_t) 65535;
    if ( new_max <= h->max_part ) return ZPIC_OK;
    if ( new_max > (uint64_t) INT32_MAX ) return fail( ZPIC_E_NOMEM, "particle buffer would exceed 2^31 particles" );
    CK( cudaStreamSynchronize( s->stream ) );
    if ( s->plan.built && s->plan.side ) CK( cudaStreamSynchronize( s->plan.side ) );
    SpDev & d = h->d;
    const size_t old = h->max_part;
    PartArrays A{}, B{};
    int * idx = nullptr; int * aux = nullptr; int * aux2 = nullptr;
    int rc = alloc_arrays( A, new_max );
    if ( rc == ZPIC_OK ) rc = alloc_arrays( B, new_max );
    if ( rc == ZPIC_OK ) rc = dalloc( &idx, new_max );
    if ( rc == ZPIC_OK ) rc = dalloc( &aux, new_max );
    if ( rc == ZPIC_OK ) rc = dalloc( &aux2, new_max );
    if ( rc != ZPIC_OK ) {
        PartArrays * na[2] = { &A, &B };
        for ( auto * a : na ) { dfree( a->cell ); dfree( a->xx ); dfree( a->xy ); dfree( a->ux ); dfree( a->uy ); dfree( a->uz ); }
        dfree( idx ); dfree( aux ); dfree( aux2 );
        return rc;
    }
    const size_t w = old * sizeof( float );
    PartArrays * src[2] = { &d.A, &d.B }, * dst[2] = { &A, &B };
    for ( int k = 0; k < 2; k++ ) {
        CK( cudaMemcpyAsync( dst[k]->cell, src[k]->cell, w, cudaMemcpyDeviceToDevice, s->stream ) );
        CK( cudaMemcpyAsync( dst[k]->xx, src[k]->xx, w, cudaMemcpyDeviceToDevice, s->stream ) );
        CK( cudaMemcpyAsync( dst[k]->xy, src[k]->xy, w, cudaMemcpyDeviceToDevice, s->stream ) );
        CK( cudaMemcpyAsync( dst[k]->ux, src[k]->ux, w, cudaMemcpyDeviceToDevice, s->stream ) );
        CK( cudaMemcpyAsync( dst[k]->uy, src[k]->uy, w, cudaMemcpyDeviceToDevice, s->stream ) );
        CK( cudaMemcpyAsync( dst[k]->uz, src[k]->uz, w, cudaMemcpyDeviceToDevice, s->stream ) );
    }
    CK( cudaMemcpyAsync( idx, d.idx, old * sizeof( int ), cudaMemcpyDeviceToDevice, s->stream ) );
    CK( cudaStreamSynchronize( s->stream ) );
    PartArrays * olds[2] = { &d.A, &d.B };
    for ( auto * a : olds ) { dfree( a->cell ); dfree( a->xx ); dfree( a->xy ); dfree( a->ux ); dfree( a->uy ); dfree( a->uz ); }
    dfree( d.idx ); dfree( d.aux ); dfree( d.aux2 );
    d.A = A; d.B = B; d.idx = idx; d.aux = aux; d.aux2 = aux2;
    d.max_part = (int) new_max;
    h->max_part = (uint32_t) new_max;
    h->grows++;
    // the descriptor copies of this simulation's plan
    Plan & P = s->plan;
    if ( P.built ) {
        for ( size_t i = 0; i < P.sps_h.size(); i++ ) {
            if ( P.sp_local[i] >= 0 && P.sp_local[i] < (int) s->species.size() && s->species[ P.sp_local[i] ] == h ) {
                SpDev v = d;
                v.run = P.sps_h[i].run;
                v.nchunk = P.sps_h[i].nchunk;
                v.chunk_target = P.sps_h[i].chunk_target;
                P.sps_h[i] = v;
                CK( cudaMemcpyAsync( P.sps_d + i, &P.sps_h[i], sizeof( SpDev ), cudaMemcpyHostToDevice, s->stream ) );
            }
        }
        CK( cudaStreamSynchronize( s->stream ) );
    }
    s->layout_gen++;
    return ZPIC_OK;
}

static void species_params( zpic_sim * s, HSpecies * sp ) {
    SpDev & d = sp->d;
    d.alpha = 0.5 * sp->dt / sp->m_q;                  // species.cpp:2305
    d.dt_dx = sp->dt / sp->dx[0]; d.dt_dy = sp->dt / sp->dx[1];
    d.q = sp->q;
    d.qnx = sp->q * sp->dx[0] / sp->dt; d.qny = sp->q * sp->dx[1] / sp->dt;
    {
        // Every current contribution of one particle segment is bounded by
        // 1.25 |q| (|v| < c, shape weights <= 1), so with |q| < 2^e the
        // fixed-point scale 2^(30-e) keeps it below 2^31 in magnitude.
        int e = 0;
        if ( sp->q != 0.0f ) std::frexp( std::fabs( sp->q ), &e );
        d.jscale = std::ldexp( 1.0f, 30 - e );
        d.jscale_inv = std::ldexp( 1.0, e - 30 );
    }
    d.perx = sp->bc[0] == ZPIC_SPECIES_BC_PERIODIC;
    d.pery = sp->bc[2] == ZPIC_SPECIES_BC_PERIODIC;
    for ( int k = 0; k < 4; k++ ) d.bc[k] = sp->bc[k];
    d.min_slack = std::max<int>( 16, (int) ( sp->ppc[0] * sp->ppc[1] * s->nxx * s->nxy / 8 ) );
    d.pool_frac = (float) s->pool_frac;
    d.reloc_room = (float) s->reloc_room;
    d.run = 0;
}

static zbhost::TileGeom geom( zpic_sim * s ) { return { s->ntx, s->nty, s->nxx, s->nxy }; }

static zbhost::Injector injector( zpic_sim * s, HSpecies * sp ) {
    zbhost::Injector I;
    I.dens = sp->dens;
    I.ppc[0] = sp->ppc[0]; I.ppc[1] = sp->ppc[1];
    I.dx[0] = sp->dx[0]; I.dx[1] = sp->dx[1];
    I.motion = sp->mw.motion();
    I.g = geom( s );
    return I;
}

static InjRule inj_rule( zpic_sim * s, HSpecies * sp, const unsigned range[4] ) {
    zbhost::Injector I = injector( s, sp );
    InjRule r{};
    r.type = sp->dens.type; r.diry = sp->dens.dir != 0;
    I.rule_params( r.a, r.b, r.cx, r.cy, r.r2 );
    r.dxx = sp->dx[0]; r.dxy = sp->dx[1];
    r.ppcx = sp->ppc[0]; r.ppcy = sp->ppc[1];
    for ( int k = 0; k < 4; k++ ) r.range[k] = range[k];
    r.tx_limit = I.tx_limit();
    return r;
}

// ---------------------------------------------------------------------------
// species advance pieces (single simulation)
// ---------------------------------------------------------------------------
static int species_index( zpic_sim * s, int sp ) {
    if ( sp < 0 || sp >= (int) s->species.size() ) return fail( ZPIC_E_INVALID, "invalid species index" );
    return ZPIC_OK;
}

// Launch the particle kernel for one species of a single simulation (no host
// synchronisation; errors surface at the next synchronising call).
static int species_kernel( zpic_sim * s, int sp, int push, int move, const int * shifts ) {
    TRY( ensure_plan( s ) );
    HSpecies * h = s->species[sp];
    if ( h->counters_dirty && move ) {
        DEV( cudaMemsetAsync( h->d.cnt, 0, 9 * (size_t) h->ntiles * sizeof( int ), s->stream ) );
        DEV( cudaMemsetAsync( h->d.nidx, 0, h->ntiles * sizeof( int ), s->stream ) );
    }
    Plan & P = s->plan;
    {
        PhaseScope ps( s, s->stream, PH_PARTICLES, 1 );
        DEV( launch_particles( s->stream, push ? 1 + h->push_type : 0, move, move ? 1 : 0,
                              P.spk1_d + P.sp_k1_off[sp], P.sp_k1_n[sp], P.sps_d, P.runs_d, shifts, P.max_tile_vol,
                              P.jacc, P.tile_n ) );
    }
    if ( move ) { h->sort_pending = true; h->counters_dirty = true; }
    if ( push ) h->energy_items = h->ntiles * P.sps_h[sp].nchunk;
    if ( move == 2 ) s->jdep_clean = false;
    return ZPIC_OK;
}

static int species_sort( zpic_sim * s, int sp, int use_extra ) {
    TRY( ensure_plan( s ) );
    HSpecies * h = s->species[sp];
    Plan & P = s->plan;
    if ( !h->sort_pending ) {
        // leaver lists are stale: detect them now (bnd_check, particles.cpp:212-303)
        DEV( cudaMemsetAsync( h->d.cnt, 0, 9 * (size_t) h->ntiles * sizeof( int ), s->stream ) );
        DEV( cudaMemsetAsync( h->d.nidx, 0, h->ntiles * sizeof( int ), s->stream ) );
        PhaseScope ps( s, s->stream, PH_SORT, 1 );
        DEV( launch_particles( s->stream, 0, 0, 1, P.spk1_d + P.sp_k1_off[sp], P.sp_k1_n[sp], P.sps_d, P.runs_d,
                              nullptr, P.max_tile_vol, 0, 0 ) );
    }
    {
        PhaseScope ps( s, s->stream, PH_SORT, 4 );
        DEV( launch_sort( s->stream, P.sort_items_d + P.sp_sort_off[sp], P.sp_sort_n[sp], P.sps_d,
                         P.splist_d + sp, 1, P.runs_d, use_extra, P.rlist_d ) );
    }
    h->sort_pending = false;
    h->counters_dirty = false;
    return ZPIC_OK;
}

// Species::advance_mov_window (species.cpp:2083-2128) for one species
// The particle kernel of a moving-window species step; *moving tells
// whether this step shifts the species' window (then the kernel shifts the
// particles by one cell).
static int mw_species_kernel( zpic_sim * s, int sp, bool * moving ) {
    HSpecies * h = s->species[sp];
    TRY( ensure_plan( s ) );
    const float t = ( h->iter + 1 ) * h->dt;        // int * float, as in the reference
    *moving = h->mw.needs_move( t );
    return species_kernel( s, sp, 1, 2, *moving ? s->shifts_d : nullptr );
}

// The rest of it: injection of the new column when the window moves, tile sort.
static int mw_species_finish( zpic_sim * s, int sp, bool moving ) {
    HSpecies * h = s->species[sp];
    if ( moving ) {
        const unsigned gx = s->ntx * s->nxx, gy = s->nty * s->nxy;
        const unsigned range[4] = { gx - 1, gx - 1, 0, gy - 1 };
        InjRule r = inj_rule( s, h, range );
        // host-side upper bound of the particle count: at most a full
        // column of cells is injected per move
        const uint64_t add = h->dens.type == ZPIC_DENSITY_NONE ? 0 : (uint64_t) gy * h->ppc[0] * h->ppc[1];
        h->np_bound += add;
        if ( capacity_for( h, h->np_bound ) > h->max_part ) {
            // the bound is loose once particles leave; read the real count
            unsigned long long st2[2];
            DEV( launch_np_stats( s->stream, s->plan.sps_d, sp, (unsigned long long *) s->dscratch ) );
            CK( cudaMemcpyAsync( st2, s->dscratch, sizeof( st2 ), cudaMemcpyDeviceToHost, s->stream ) );
            CK( cudaStreamSynchronize( s->stream ) );
            h->np_bound = st2[0] + add;
            // still short: grow (by a quarter at least, so that a steadily
            // injecting run grows rarely)
            if ( capacity_for( h, h->np_bound ) > h->max_part )
                TRY( species_grow( s, h, std::max<uint64_t>( capacity_for( h, h->np_bound ),
                                                             (uint64_t) h->max_part + h->max_part / 4 ) ) );
        }
        if ( h->dens.type != ZPIC_DENSITY_NONE ) {
            // the window-dependent rule parameters come from the device's move count
            DEV( launch_inj_dyn( s->stream, h->inj_dyn, h->mw_nmove_d, h->dens.type, h->dens.a, h->dens.b,
                                 h->dx[0], h->mw.dx ) );
            r.dyn = h->inj_dyn;
            DEV( cudaMemsetAsync( h->d.extra, 0, h->ntiles * sizeof( int ), s->stream ) );
            DEV( launch_inject( s->stream, sp, range[0] / s->nxx, range[1] / s->nxx, range[2] / s->nxy, range[3] / s->nxy,
                                s->plan.sps_d, s->plan.runs_d, r, 1 ) );
            s->launches += 2;
        }
        TRY( species_sort( s, sp, h->dens.type != ZPIC_DENSITY_NONE ) );
        if ( h->dens.type != ZPIC_DENSITY_NONE ) {
            DEV( launch_inject( s->stream, sp, range[0] / s->nxx, range[1] / s->nxx, range[2] / s->nxy, range[3] / s->nxy,
                                s->plan.sps_d, s->plan.runs_d, r, 0 ) );
            s->launches++;
        }
        h->mw.advance();
    } else {
        TRY( species_sort( s, sp, 0 ) );
    }
    h->iter++;
    return ZPIC_OK;
}

static int species_advance_mw( zpic_sim * s, int sp ) {
    bool moving = false;
    TRY( mw_species_kernel( s, sp, &moving ) );
    return mw_species_finish( s, sp, moving );
}

// ---- autotuning of CTAs per tile ----
// Candidates: the automatic choices (0 uniform, -1 occupancy-balanced) and
// 1, 2, 4, ... 64 CTAs per tile, keeping at least 256 particles per CTA on
// average.  Each candidate runs one
// untimed step (graph capture) and `steps` timed steps; the trial steps are
// real steps of the simulation(s).  The physics does not depend on the
// choice; only the order in which the per-CTA partial currents are added to
// the raw current (FP32) does.
static std::vector<int> chunk_candidates( uint64_t particles, uint64_t tiles, int automatic ) {
    std::vector<int> c;
    const double per_tile = tiles ? (double) particles / tiles : 0.0;
    for ( int k = 1; k <= 64; k *= 2 )
        if ( k == 1 || per_tile / k >= 256.0 ) c.push_back( k );
    (void) automatic;
    c.insert( c.begin(), -1 );
    c.insert( c.begin(), 0 );
    return c;
}

template < class Advance >
static int time_candidate( cudaStream_t st, int steps, Advance adv, float * ms ) {
    cudaEvent_t e0, e1;
    CK( cudaEventCreate( &e0 ) ); CK( cudaEventCreate( &e1 ) );
    int rc = adv( 1 );
    if ( rc == ZPIC_OK ) {
        CK( cudaEventRecord( e0, st ) );
        rc = adv( steps );
        CK( cudaEventRecord( e1, st ) );
        CK( cudaEventSynchronize( e1 ) );
        CK( cudaEventElapsedTime( ms, e0, e1 ) );
    }
    cudaEventDestroy( e0 ); cudaEventDestroy( e1 );
    return rc;
}

static uint64_t particles_of( zpic_sim * s ) {
    uint64_t n = 0;
    for ( auto * h : s->species ) n += h->np_bound;
    return n;
}

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
extern "C" {

const char * zpic_b200_last_error( void ) { return g_err.c_str(); }
int zpic_b200_version( void ) { return 10000; }

int zpic_b200_set_device( int device ) {
    int n = 0;
    CK( cudaGetDeviceCount( &n ) );
    if ( device < 0 || device >= n ) return fail( ZPIC_E_INVALID, "invalid device" );
    g_device = device;
    return ZPIC_OK;
}

int zpic_b200_sim_create( uint32_t ntx, uint32_t nty, uint32_t nxx, uint32_t nxy,
                          float boxx, float boxy, double dt, zpic_sim ** out ) {
    if ( !out ) return fail( ZPIC_E_INVALID, "null output" );
    *out = nullptr;
    if ( ntx == 0 || nty == 0 ) return fail( ZPIC_E_INVALID, "Invalid number of tiles" );      // grid.h:34-38
    if ( nxx == 0 || nxy == 0 ) return fail( ZPIC_E_INVALID, "Invalid tile size" );            // grid.h:40-43
    {
        // every tile kernel stages whole tiles in shared memory (227 KB per block)
        const int tv = roundup4( ( nxx + 3 ) * ( nxy + 3 ) );
        const size_t need = std::max( particle_smem_bytes( tv, 1 ), yee_smem_bytes( tv ) );
        if ( nxx > 1024 || nxy > 1024 || need > 227 * 1024 )
            return fail( ZPIC_E_INVALID, "tile too large: its field tiles do not fit in shared memory" );
    }
    // Courant condition (emf.cpp:20-28)
    const float dxx = boxx / ( nxx * ntx ), dxy = boxy / ( nxy * nty );
    const float cour = std::sqrt( 1.0f / ( 1.0f / ( dxx * dxx ) + 1.0f / ( dxy * dxy ) ) );
    if ( dt >= cour ) {
        char m[160];
        snprintf( m, sizeof m, "Invalid timestep, courant condition violation: the maximum timestep is dt = %g", cour );
        return fail( ZPIC_E_INVALID, m );
    }
    int dev = g_device;
    if ( dev < 0 ) CK( cudaGetDevice( &dev ) );
    CK( cudaSetDevice( dev ) );
    auto s = std::make_unique<zpic_sim>();
    s->device = dev;
    s->ntx = ntx; s->nty = nty; s->nxx = nxx; s->nxy = nxy;
    s->box[0] = boxx; s->box[1] = boxy; s->dt = dt;
    s->dx[0] = dxx; s->dx[1] = dxy;
    CK( cudaStreamCreateWithFlags( &s->stream, cudaStreamNonBlocking ) );
    RunDev & R = s->run;
    R.ntx = ntx; R.nty = nty; R.nxx = nxx; R.nxy = nxy;
    R.extx = 1 + nxx + 2; R.exty = 1 + nxy + 2;
    R.gc_off = 1 * R.extx + 1;
    R.tile_vol = roundup4( R.extx * R.exty );
    const float dtx = dt / dxx, dty = dt / dxy;                 // emf.cpp:524-525
    R.dtx = dtx; R.dty = dty; R.dtx2 = dtx / 2; R.dty2 = dty / 2;
    R.dt = (float) dt;
    const size_t nf = s->grid_floats();
    TRY( dalloc( &R.E, nf ) ); TRY( dalloc( &R.B, nf ) ); TRY( dalloc( &R.J, nf ) ); TRY( dalloc( &R.Jdep, nf ) );
    TRY( dalloc( &R.bcol, (size_t) ntx * nty * nxy * 3 ) );
    CK( cudaMemset( R.E, 0, nf * sizeof( float ) ) );
    CK( cudaMemset( R.B, 0, nf * sizeof( float ) ) );
    CK( cudaMemset( R.J, 0, nf * sizeof( float ) ) );
    CK( cudaMemset( R.Jdep, 0, nf * sizeof( float ) ) );
    TRY( dalloc( &s->status, 1 ) );
    CK( cudaMemset( s->status, 0, sizeof( int ) ) );
    R.status = s->status;
    R.wait_limit = WAIT_LIMIT_DEFAULT;
    TRY( dalloc( &s->dscratch, 64 ) );
    CK( cudaMallocHost( (void **) &s->hscratch, 64 * sizeof( double ) ) );
    // cell shift of a moving-window step: -1 for whichever species the
    // particle kernel is launched for (at most MAX_SPECIES per simulation)
    TRY( dalloc( &s->shifts_d, MAX_SPECIES ) );
    {
        std::vector<int> neg( MAX_SPECIES, -1 );
        CK( cudaMemcpy( s->shifts_d, neg.data(), MAX_SPECIES * sizeof( int ), cudaMemcpyHostToDevice ) );
    }
    TRY( upload_run( s.get() ) );
    *out = s.release();
    return ZPIC_OK;
}

int zpic_b200_sim_destroy( zpic_sim * s ) {
    if ( !s ) return ZPIC_OK;
    cudaSetDevice( s->device );
    cudaStreamSynchronize( s->stream );
    resolve_phase_events( s );
    s->plan.release();
    for ( auto * sp : s->species ) { sp->free_all(); delete sp; }
    dfree( s->run.E ); dfree( s->run.B ); dfree( s->run.J ); dfree( s->run.Jdep ); dfree( s->run.bcol );
    dfree( s->status ); dfree( s->dscratch ); dfree( s->shifts_d ); dfree( s->fe_part_d );
    if ( s->fe_part_h ) { cudaFreeHost( s->fe_part_h ); s->fe_part_h = nullptr; }
    if ( s->hscratch ) cudaFreeHost( s->hscratch );
    cudaStreamDestroy( s->stream );
    delete s;
    return ZPIC_OK;
}

int zpic_b200_sim_add_species( zpic_sim * s, const zpic_species_desc * desc, int32_t * species_id ) {
    TRY( sim_select( s ) );
    if ( !desc ) return fail( ZPIC_E_INVALID, "null species description" );
    if ( desc->m_q == 0 ) return fail( ZPIC_E_INVALID, "Invalid m_q value, must be not 0" );          // species.cpp:1698
    if ( s->species.size() >= (size_t) MAX_SPECIES ) return fail( ZPIC_E_INVALID, "too many species" );
    if ( desc->ppc[0] < 1 || desc->ppc[1] < 1 ) return fail( ZPIC_E_INVALID, "Invalid ppc value, must be >= 1 in all directions" );
    if ( desc->density.type < 0 || desc->density.type > 4 ) return fail( ZPIC_E_INVALID, "invalid density type" );
    if ( desc->udist.type < 0 || desc->udist.type > 3 ) return fail( ZPIC_E_INVALID, "invalid udist type" );
    if ( desc->udist.type == ZPIC_UDIST_THERMALCORR && desc->udist.npmin <= 1 )
        return fail( ZPIC_E_INVALID, "invalid npmin parameter, must be > 1" );                        // udist.h:47-50
    for ( int a = 0; a < 2; a++ ) {                                                                     // species.h:211-235
        const int lo = desc->bc[2*a], hi = desc->bc[2*a+1];
        if ( ( lo == ZPIC_SPECIES_BC_PERIODIC || hi == ZPIC_SPECIES_BC_PERIODIC ) && lo != hi )
            return fail( ZPIC_E_INVALID, "Species boundary type mismatch" );
    }
    if ( s->species.size() >= 32 ) return fail( ZPIC_E_INVALID, "too many species" );
    s->plan.release();
    auto sp = std::make_unique<HSpecies>();
    sp->name = desc->name ? desc->name : "species";
    sp->m_q = desc->m_q;
    sp->ppc[0] = desc->ppc[0]; sp->ppc[1] = desc->ppc[1];
    sp->dens = desc->density;
    sp->ud = desc->udist;
    sp->push_type = desc->push_type ? 1 : 0;
    for ( int k = 0; k < 4; k++ ) sp->bc[k] = desc->bc[k];
    // Species::initialize (species.cpp:1730-1788)
    sp->box[0] = s->box[0]; sp->box[1] = s->box[1];
    sp->dt = (float) s->dt;
    sp->id = (int) s->species.size() + 1;                          // simulation.h:68-71
    const float n0 = sp->dens.type == ZPIC_DENSITY_NONE ? 0.f : std::fabs( sp->dens.n0 );
    sp->q = std::copysign( n0, sp->m_q ) / ( sp->ppc[0] * sp->ppc[1] );
    const float dimsx = (float) ( s->nxx * s->ntx ), dimsy = (float) ( s->nxy * s->nty );
    sp->dx[0] = sp->box[0] / dimsx; sp->dx[1] = sp->box[1] / dimsy;
    const uint64_t ref_max = (uint64_t) ( s->capacity_factor * dimsx * dimsy * sp->ppc[0] * sp->ppc[1] );
    const int nt = s->ntx * s->nty;
    // initial particles on the host, reference algorithms and order
    zbhost::Injector I = injector( s, sp.get() );
    const unsigned range[4] = { 0, (unsigned) ( s->nxx * s->ntx - 1 ), 0, (unsigned) ( s->nxy * s->nty - 1 ) };
    std::vector<int> np_inj( nt, 0 ), offset( nt, 0 ), np( nt, 0 );
    I.count( range, np_inj.data() );
    long long total = 0;
    for ( int t = 0; t < nt; t++ ) { offset[t] = (int) total; total += np_inj[t]; }
    std::vector<int32_t> ix( 2 * total ); std::vector<float> x( 2 * total ), u( 3 * total );
    I.inject( range, offset.data(), np.data(), ix.data(), x.data(), u.data() );
    zbhost::udist_set( sp->ud, sp->id, geom( s ), offset.data(), np.data(), ix.data(), u.data() );
    // capacity: the reference's max_part, raised if the slot layout needs more
    const int min_slack = std::max<int>( 16, (int) ( sp->ppc[0] * sp->ppc[1] * s->nxx * s->nxy / 8 ) );
    uint64_t need = 0; for ( int t = 0; t < nt; t++ ) need += roundup4( np[t] );
    const uint64_t max_part = std::max<uint64_t>( { ref_max, need + (uint64_t) nt * 4, 1024 } );
    (void) min_slack;
    TRY( species_alloc( s, sp.get(), max_part ) );
    species_params( s, sp.get() );
    sp->d.nchunk = 1;
    TRY( dalloc( &sp->d.energy, (size_t) nt * 64 ) );
    CK( cudaMemset( sp->d.energy, 0, (size_t) nt * 64 * sizeof( double ) ) );
    HSpecies * raw = sp.get();
    s->species.push_back( sp.release() );
    // chunking depends on the total tile count of all species
    int ntot = 0; for ( auto * h : s->species ) ntot += h->ntiles;
    TRY( species_upload( s, raw, np, ix.data(), x.data(), u.data() ) );
    set_chunks( s );
    if ( species_id ) *species_id = (int) s->species.size() - 1;
    return ZPIC_OK;
}

int zpic_b200_sim_set_moving_window( zpic_sim * s ) {
    TRY( sim_select( s ) );
    // Simulation::set_moving_window (simulation.h:56-62): each object checks iter == 0
    if ( s->emf_iter == 0 ) {
        s->emf_mw.init( s->dx[0] );
        s->emf_bc[0] = s->emf_bc[1] = ZPIC_EMF_BC_NONE;
    }
    if ( s->cur_iter == 0 ) {
        s->cur_mw.init( s->dx[0] );
        s->cur_bc[0] = s->cur_bc[1] = ZPIC_CURRENT_BC_NONE;
    }
    for ( auto * sp : s->species ) {
        if ( sp->iter == 0 ) {
            sp->mw.init( sp->dx[0] );
            sp->bc[0] = sp->bc[1] = ZPIC_SPECIES_BC_OPEN;
            species_params( s, sp );
        }
    }
    TRY( upload_run( s ) );
    return ZPIC_OK;
}

int zpic_b200_sim_set_option( zpic_sim * s, const char * key, double v ) {
    TRY( sim_select( s ) );
    if ( !key ) return fail( ZPIC_E_INVALID, "null option" );
    std::string k( key );
    if ( k == "graph" ) { s->use_graph = v != 0; }
    else if ( k == "profile" ) {
        // 1: events around each phase, steps issued eagerly; 2: events
        // around the particle phase as nodes of the step graph, so that graph
        // replays are timed
        const int m = (int) v;
        if ( m < 0 || m > 2 || m != v ) return fail( ZPIC_E_INVALID, "profile must be 0, 1 or 2" );
        s->profile = m;
        if ( m == 1 ) s->use_graph = false;
    }
    else if ( k == "jacc" ) {
        const int j = (int) v;
        if ( j < 0 || j > 2 || j != v ) return fail( ZPIC_E_INVALID, "jacc must be 0, 1 or 2" );
        if ( j != s->jacc ) { s->jacc = j; s->plan.release(); }
    }
    else if ( k == "reorder" ) {
        const int r = (int) v;
        if ( r < 0 || r != v ) return fail( ZPIC_E_INVALID, "reorder must be a step count >= 0" );
        s->reorder_every = r;
        s->plan.release();
    }
    else if ( k == "capacity_factor" ) {
        // initial particle-buffer capacity of species added afterwards, in
        // particles per cell per ppc (buffers grow when they run short)
        if ( !( v > 0 && v <= 64 ) ) return fail( ZPIC_E_INVALID, "capacity_factor must be in (0, 64]" );
        s->capacity_factor = v;
    }
    else if ( k == "pool_fraction" || k == "relocation_room" ) {
        // tile-slot policy: the share of the free capacity kept as a pool at
        // the end of the buffer (tiles that outgrow their slots move there),
        // and the room a moved tile gets, as a share of its count
        if ( !( v >= 0 && v <= ( k == "pool_fraction" ? 0.95 : 16.0 ) ) ) return fail( ZPIC_E_INVALID, k + " out of range" );
        if ( k == "pool_fraction" ) s->pool_frac = v; else s->reloc_room = v;
        for ( auto * h : s->species ) species_params( s, h );
        s->plan.release();
        s->layout_gen++;
    }
    else if ( k == "wait_limit" ) {
        // polls of the kernels' bounded waits on their bulk copies before
        // they give up (default ~0.5 s worth)
        const int w = (int) v;
        if ( w < 1 || w != v ) return fail( ZPIC_E_INVALID, "wait_limit must be a poll count >= 1" );
        s->run.wait_limit = w;
        TRY( upload_run( s ) );
    }
    else if ( k == "chunks" ) {
        // the per-item energy array holds 64 chunks per tile
        s->chunks_opt = std::min( 64, std::max( -1, (int) v ) );
        set_chunks( s );
        s->plan.release();
    }
    else return fail( ZPIC_E_INVALID, "unknown option " + k );
    return ZPIC_OK;
}

int zpic_b200_sim_advance( zpic_sim * s, int32_t nsteps ) {
    TRY( sim_select( s ) );
    if ( nsteps < 0 ) return fail( ZPIC_E_INVALID, "negative step count" );
    TRY( ensure_plan( s ) );
    // pending fine-grained work must not be mixed with a full step
    for ( auto * sp : s->species ) {
        if ( sp->counters_dirty ) {
            CK( cudaMemsetAsync( sp->d.cnt, 0, 9 * (size_t) sp->ntiles * sizeof( int ), s->stream ) );
            CK( cudaMemsetAsync( sp->d.nidx, 0, sp->ntiles * sizeof( int ), s->stream ) );
            sp->counters_dirty = false;
        }
    }
    uint64_t l = 0;
    TRY( plan_advance( s->plan, s->stream, nsteps, s->use_graph && s->profile != 1, &l ) );
    s->launches += l;
    return ZPIC_OK;
}

// One Simulation::advance_mov_window step (simulation.h:113-130): species,
// current, fields and the window shift.  After the particle kernels the
// species' injection and sort (particle arrays only) stay on the
// simulation's stream while current, fields and the field shift (grids only)
// run on the plan's side stream; the two join before the step ends.
static int mw_step( zpic_sim * s ) {
    TRY( ensure_jdep_clean( s, s->stream ) );
    TRY( ensure_plan( s ) );
    s->j_final = false;
    const size_t nsp = s->species.size();
    std::vector<char> moving( nsp, 0 );
    for ( size_t k = 0; k < nsp; k++ ) {
        bool m = false;
        TRY( mw_species_kernel( s, (int) k, &m ) );
        moving[k] = m;
    }
    Plan & P = s->plan;
    DEV( cudaEventRecord( P.fork, s->stream ) );
    DEV( cudaStreamWaitEvent( P.side, P.fork, 0 ) );
    TRY( run_current( P, P.side ) );
    s->cur_iter++;
    if ( s->cur_mw.needs_move( s->cur_iter * s->dt ) ) s->cur_mw.advance();
    // a window shift right after the field solve is folded into it (the Yee
    // kernel writes its tiles shifted, one guard refresh completes the shift)
    // when no physical boundary has to be applied in between and every y
    // guard cell has a source (periodic y): then every field value, guard
    // cells included, comes out as with the solve and the shift one after
    // the other
    const bool shift = s->emf_mw.active && s->emf_mw.needs_move( ( s->emf_iter + 1 ) * s->dt );
    bool fused = shift && P.sims.size() == 1 && s->run.emf_pery;
    for ( int k = 0; k < 4; k++ ) fused = fused && s->emf_bc[k] <= ZPIC_EMF_BC_PERIODIC;
    TRY( run_fields( P, P.side, 1, 0, 1, fused ) );
    s->jdep_clean = true;
    s->j_final = true;
    s->emf_iter++;
    if ( shift ) {
        if ( !fused ) TRY( run_shift( P, P.side, 0 ) );
        s->emf_mw.advance();
    }
    DEV( cudaEventRecord( P.join, P.side ) );
    for ( size_t k = 0; k < nsp; k++ ) TRY( mw_species_finish( s, (int) k, moving[k] != 0 ) );
    DEV( cudaStreamWaitEvent( s->stream, P.join, 0 ) );
    s->iter++;
    return ZPIC_OK;
}

// Moving-window steps replay CUDA graphs: the device work of a step depends
// only on which windows move in it (the window-dependent injection
// parameters are computed on the device), so one graph per pattern of moves
// is captured the first time it occurs.  Replays run the step's host code
// once more with device work suppressed, for its bookkeeping.  Steps in which
// a species' particle bound must be checked against the device (a host
// synchronisation) run without a graph.
int zpic_b200_sim_advance_mov_window( zpic_sim * s, int32_t nsteps ) {
    TRY( sim_select( s ) );
    TRY( ensure_plan( s ) );
    for ( int n = 0; n < nsteps; n++ ) {
        unsigned key = 0;
        bool eager = !s->use_graph || s->profile || !s->jdep_clean || s->species.size() > 30;
        const unsigned gy = s->nty * s->nxy;
        for ( size_t k = 0; k < s->species.size() && !eager; k++ ) {
            HSpecies * h = s->species[k];
            if ( h->counters_dirty || h->sort_pending ) eager = true;
            if ( h->mw.needs_move( (float) ( ( h->iter + 1 ) * h->dt ) ) ) {
                key |= 1u << k;
                const uint64_t add = h->dens.type == ZPIC_DENSITY_NONE ? 0 : (uint64_t) gy * h->ppc[0] * h->ppc[1];
                if ( capacity_for( h, h->np_bound + add ) > h->max_part ) eager = true;
            }
        }
        if ( s->emf_mw.active && s->emf_mw.needs_move( ( s->emf_iter + 1 ) * s->dt ) ) key |= 1u << 31;
        if ( eager ) {
            TRY( mw_step( s ) );
            uint64_t l = 0;
            TRY( maybe_reorder( s->plan, s->stream, &l ) );
            s->launches += l;
            continue;
        }
        Plan & P = s->plan;
        const uint64_t l0 = s->launches;
        auto it = P.mw_graphs.find( key );
        if ( it == P.mw_graphs.end() ) {
            cudaGraph_t g;
            CK( cudaStreamBeginCapture( s->stream, cudaStreamCaptureModeThreadLocal ) );
            const int rc = mw_step( s );
            const cudaError_t e = cudaStreamEndCapture( s->stream, &g );
            if ( rc != ZPIC_OK ) return rc;
            if ( e != cudaSuccess ) return fail( ZPIC_E_CUDA, std::string( "graph capture: " ) + cudaGetErrorString( e ) );
            cudaGraphExec_t ge;
            const int nk = count_graph_kernels( g );
            const cudaError_t e2 = cudaGraphInstantiate( &ge, g, 0 );
            cudaGraphDestroy( g );
            if ( e2 != cudaSuccess ) return fail( ZPIC_E_CUDA, std::string( "graph instantiate: " ) + cudaGetErrorString( e2 ) );
            it = P.mw_graphs.emplace( key, std::make_pair( ge, nk ) ).first;
        } else {
            g_dry = true;
            const int rc = mw_step( s );
            g_dry = false;
            if ( rc != ZPIC_OK ) return rc;
        }
        CK( cudaGraphLaunch( it->second.first, s->stream ) );
        s->launches = l0 + it->second.second;
        uint64_t l = 0;
        TRY( maybe_reorder( P, s->stream, &l ) );
        s->launches += l;
    }
    return ZPIC_OK;
}

int zpic_b200_sim_iter( zpic_sim * s, uint32_t * iter ) {
    if ( !s || !iter ) return fail( ZPIC_E_INVALID, "null argument" );
    *iter = s->iter;
    return ZPIC_OK;
}

int zpic_b200_sim_synchronize( zpic_sim * s ) {
    TRY( sim_select( s ) );
    CK( cudaStreamSynchronize( s->stream ) );
    return check_status( s );
}

int zpic_b200_sim_phase_times( zpic_sim * s, double * ms, uint64_t * launches, int32_t n ) {
    TRY( sim_select( s ) );
    resolve_phase_events( s );
    for ( int p = 0; p < n && p < PH_N; p++ ) {
        if ( ms ) ms[p] = s->phase_ms[p];
        if ( launches ) launches[p] = s->phase_launches[p];
    }
    return ZPIC_OK;
}

int zpic_b200_sim_reset_phase_times( zpic_sim * s ) {
    TRY( sim_select( s ) );
    resolve_phase_events( s );
    for ( int p = 0; p < PH_N; p++ ) { s->phase_ms[p] = 0; s->phase_launches[p] = 0; }
    return ZPIC_OK;
}

int zpic_b200_sim_launch_count( zpic_sim * s, uint64_t * count ) {
    if ( !s || !count ) return fail( ZPIC_E_INVALID, "null argument" );
    *count = s->launches;
    return ZPIC_OK;
}

int zpic_b200_sim_stream( zpic_sim * s, void ** stream ) {
    if ( !s || !stream ) return fail( ZPIC_E_INVALID, "null argument" );
    *stream = (void *) s->stream;
    return ZPIC_OK;
}

// ---- EMF ----
int zpic_b200_emf_set_bc( zpic_sim * s, const int32_t bc[4] ) {
    TRY( sim_select( s ) );
    for ( int a = 0; a < 2; a++ )                                   // emf.h:113-130
        if ( ( bc[2*a] == ZPIC_EMF_BC_PERIODIC || bc[2*a+1] == ZPIC_EMF_BC_PERIODIC ) && bc[2*a] != bc[2*a+1] )
            return fail( ZPIC_E_INVALID, "EMF boundary type mismatch" );
    for ( int k = 0; k < 4; k++ ) s->emf_bc[k] = bc[k];
    return upload_run( s );
}

int zpic_b200_emf_advance( zpic_sim * s, int32_t with_current ) {
    TRY( sim_select( s ) );
    TRY( ensure_plan( s ) );
    TRY( run_fields( s->plan, s->stream, with_current ? 1 : 0, s->j_final ? 0 : 1, 0 ) );
    s->emf_iter++;
    if ( s->emf_mw.active && s->emf_mw.needs_move( s->emf_iter * s->dt ) ) {
        TRY( run_shift( s->plan, s->stream, 0 ) );
        s->emf_mw.advance();
    }
    CK( cudaStreamSynchronize( s->stream ) );
    return check_status( s );
}

int zpic_b200_emf_energy( zpic_sim * s, double ene_E[3], double ene_B[3] ) {
    TRY( sim_select( s ) );
    TRY( ensure_plan( s ) );
    const int nt = s->ntx * s->nty;
    // partials buffers kept for the simulation's lifetime (a per-step
    // diagnostic: no allocation, no pageable copy per call)
    if ( !s->fe_part_d ) TRY( dalloc( &s->fe_part_d, 6 * (size_t) nt ) );
    if ( !s->fe_part_h ) {
        const cudaError_t e = cudaMallocHost( (void **) &s->fe_part_h, 6 * (size_t) nt * sizeof( double ) );
        if ( e != cudaSuccess ) { s->fe_part_h = nullptr; return fail( ZPIC_E_NOMEM, std::string( "cudaMallocHost: " ) + cudaGetErrorString( e ) ); }
    }
    CK( launch_field_energy( s->stream, s->plan.runs_d, 0, nt, s->fe_part_d ) );
    s->launches++;
    const double * h = s->fe_part_h;
    CK( cudaMemcpyAsync( s->fe_part_h, s->fe_part_d, 6 * (size_t) nt * sizeof( double ), cudaMemcpyDeviceToHost, s->stream ) );
    CK( cudaStreamSynchronize( s->stream ) );
    double e[6] = { 0, 0, 0, 0, 0, 0 };
    for ( int t = 0; t < nt; t++ ) for ( int k = 0; k < 6; k++ ) e[k] += h[6 * (size_t) t + k];   // tile order
    for ( int k = 0; k < 3; k++ ) { ene_E[k] = e[k]; ene_B[k] = e[3 + k]; }
    return check_status( s );
}

int zpic_b200_laser_add( zpic_sim * s, const zpic_laser_desc * l ) {
    TRY( sim_select( s ) );
    if ( !l ) return fail( ZPIC_E_INVALID, "null laser" );
    std::vector<float> E, B;
    if ( zbhost::laser_fields( *l, geom( s ), s->box, E, B ) < 0 )
        return fail( ZPIC_E_INVALID, "Invalid laser parameters" );
    float * tmp = nullptr;
    TRY( dalloc( &tmp, E.size() ) );
    CK( cudaMemcpyAsync( tmp, E.data(), E.size() * sizeof( float ), cudaMemcpyHostToDevice, s->stream ) );
    CK( launch_grid_add( s->stream, s->run.E, tmp, E.size() ) );
    CK( cudaStreamSynchronize( s->stream ) );
    CK( cudaMemcpyAsync( tmp, B.data(), B.size() * sizeof( float ), cudaMemcpyHostToDevice, s->stream ) );
    CK( launch_grid_add( s->stream, s->run.B, tmp, B.size() ) );
    CK( cudaStreamSynchronize( s->stream ) );
    s->launches += 2;
    dfree( tmp );
    return ZPIC_OK;
}

// ---- Current ----
int zpic_b200_current_set_bc( zpic_sim * s, const int32_t bc[4] ) {
    TRY( sim_select( s ) );
    for ( int a = 0; a < 2; a++ )                                   // current.h:95-112
        if ( ( bc[2*a] == ZPIC_CURRENT_BC_PERIODIC || bc[2*a+1] == ZPIC_CURRENT_BC_PERIODIC ) && bc[2*a] != bc[2*a+1] )
            return fail( ZPIC_E_INVALID, "Current boundary type mismatch" );
    for ( int k = 0; k < 4; k++ ) s->cur_bc[k] = bc[k];
    return upload_run( s );
}

int zpic_b200_current_set_filter( zpic_sim * s, int32_t type, int32_t dir, uint32_t order ) {
    TRY( sim_select( s ) );
    if ( type < 0 || type > 2 ) return fail( ZPIC_E_INVALID, "invalid filter type" );
    s->ftype = type; s->fdir = dir ? 1 : 0; s->forder = order > 0 ? order : 1;   // filter.h:35
    s->plan.built = false;
    return ZPIC_OK;
}

int zpic_b200_current_zero( zpic_sim * s ) {
    TRY( sim_select( s ) );
    s->jdep_clean = false;
    TRY( ensure_jdep_clean( s, s->stream ) );
    CK( cudaMemsetAsync( s->run.J, 0, s->grid_floats() * sizeof( float ), s->stream ) );
    s->j_final = false;
    return ZPIC_OK;
}

int zpic_b200_current_advance( zpic_sim * s ) {
    TRY( sim_select( s ) );
    TRY( ensure_plan( s ) );
    TRY( run_current( s->plan, s->stream ) );
    s->j_final = true;
    s->cur_iter++;
    if ( s->cur_mw.needs_move( s->cur_iter * s->dt ) ) s->cur_mw.advance();
    CK( cudaStreamSynchronize( s->stream ) );
    return check_status( s );
}

// ---- Species ----
int zpic_b200_species_advance( zpic_sim * s, int32_t sp, int32_t mode ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) );
    if ( mode == ZPIC_ADVANCE_FULL ) TRY( species_kernel( s, sp, 1, 2, nullptr ) );
    else if ( mode == ZPIC_ADVANCE_CURRENT ) TRY( species_kernel( s, sp, 0, 2, nullptr ) );
    else if ( mode == ZPIC_ADVANCE_FREE ) TRY( species_kernel( s, sp, 0, 1, nullptr ) );
    else return fail( ZPIC_E_INVALID, "invalid advance mode" );
    TRY( species_sort( s, sp, 0 ) );
    s->species[sp]->iter++;
    s->j_final = false;
    return ZPIC_OK;
}

int zpic_b200_species_advance_mov_window( zpic_sim * s, int32_t sp ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) );
    s->j_final = false;
    return species_advance_mw( s, sp );
}

int zpic_b200_species_push( zpic_sim * s, int32_t sp ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) );
    return species_kernel( s, sp, 1, 0, nullptr );
}

int zpic_b200_species_move( zpic_sim * s, int32_t sp ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) );
    s->j_final = false;
    return species_kernel( s, sp, 0, 2, nullptr );
}

int zpic_b200_species_process_bc( zpic_sim * s, int32_t sp ) {
    // Reflecting walls are applied inside the move kernel (after each move),
    // which is where Species::advance calls process_bc (species.cpp:2060).
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) );
    return ZPIC_OK;
}

int zpic_b200_species_tile_sort( zpic_sim * s, int32_t sp ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) );
    return species_sort( s, sp, 0 );
}

int zpic_b200_species_set_bc( zpic_sim * s, int32_t sp, const int32_t bc[4] ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) );
    for ( int a = 0; a < 2; a++ )
        if ( ( bc[2*a] == ZPIC_SPECIES_BC_PERIODIC || bc[2*a+1] == ZPIC_SPECIES_BC_PERIODIC ) && bc[2*a] != bc[2*a+1] )
            return fail( ZPIC_E_INVALID, "Species boundary type mismatch" );
    HSpecies * h = s->species[sp];
    for ( int k = 0; k < 4; k++ ) h->bc[k] = bc[k];
    species_params( s, h );
    s->plan.release();
    return ZPIC_OK;
}

int zpic_b200_species_set_push_type( zpic_sim * s, int32_t sp, int32_t type ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) );
    const int t = type ? 1 : 0;
    if ( s->species[sp]->push_type != t ) {
        s->species[sp]->push_type = t;
        s->plan.release();
    }
    return ZPIC_OK;
}

int zpic_b200_species_energy( zpic_sim * s, int32_t sp, double * energy ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) ); TRY( ensure_plan( s ) );
    HSpecies * h = s->species[sp];
    const int items = h->energy_items > 0 ? h->energy_items : h->ntiles * h->d.nchunk;
    CK( launch_energy_sum( s->stream, s->plan.sps_d, sp, items, s->dscratch ) );
    s->launches++;
    double d = 0;
    CK( cudaMemcpyAsync( &d, s->dscratch, sizeof( double ), cudaMemcpyDeviceToHost, s->stream ) );
    CK( cudaStreamSynchronize( s->stream ) );
    *energy = d * h->q * h->m_q * h->dx[0] * h->dx[1];          // species.h:365-368
    return check_status( s );
}

int zpic_b200_species_nmove( zpic_sim * s, int32_t sp, uint64_t * nmove ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) );
    unsigned long long v = 0;
    CK( cudaMemcpyAsync( &v, s->species[sp]->d.nmove, sizeof( v ), cudaMemcpyDeviceToHost, s->stream ) );
    CK( cudaStreamSynchronize( s->stream ) );
    *nmove = v;
    return ZPIC_OK;
}

int zpic_b200_species_repacks( zpic_sim * s, int32_t sp, uint64_t * repacks ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) );
    if ( !repacks ) return fail( ZPIC_E_INVALID, "null argument" );
    unsigned long long v = 0;
    CK( cudaMemcpyAsync( &v, s->species[sp]->d.nmove + 1, sizeof( v ), cudaMemcpyDeviceToHost, s->stream ) );
    CK( cudaStreamSynchronize( s->stream ) );
    *repacks = v;
    return ZPIC_OK;
}

int zpic_b200_species_relocations( zpic_sim * s, int32_t sp, uint64_t * tiles ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) );
    if ( !tiles ) return fail( ZPIC_E_INVALID, "null argument" );
    unsigned long long v = 0;
    CK( cudaMemcpyAsync( &v, s->species[sp]->d.nmove + 2, sizeof( v ), cudaMemcpyDeviceToHost, s->stream ) );
    CK( cudaStreamSynchronize( s->stream ) );
    *tiles = v;
    return ZPIC_OK;
}

int zpic_b200_species_max_part( zpic_sim * s, int32_t sp, uint32_t * max_part ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) );
    if ( !max_part ) return fail( ZPIC_E_INVALID, "null argument" );
    *max_part = s->species[sp]->max_part;
    return ZPIC_OK;
}

int zpic_b200_sim_nmove( zpic_sim * s, uint64_t * nmove ) {
    TRY( sim_select( s ) );
    uint64_t t = 0;
    for ( size_t k = 0; k < s->species.size(); k++ ) { uint64_t v; TRY( zpic_b200_species_nmove( s, (int) k, &v ) ); t += v; }
    *nmove = t;
    return ZPIC_OK;
}

static int np_stats( zpic_sim * s, int sp, unsigned long long out[2] ) {
    TRY( ensure_plan( s ) );
    CK( launch_np_stats( s->stream, s->plan.sps_d, sp, (unsigned long long *) s->dscratch ) );
    s->launches++;
    CK( cudaMemcpyAsync( out, s->dscratch, 2 * sizeof( unsigned long long ), cudaMemcpyDeviceToHost, s->stream ) );
    CK( cudaStreamSynchronize( s->stream ) );
    return ZPIC_OK;
}

int zpic_b200_species_np_total( zpic_sim * s, int32_t sp, uint64_t * np ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) );
    unsigned long long st[2]; TRY( np_stats( s, sp, st ) );
    *np = st[0];
    return ZPIC_OK;
}

int zpic_b200_species_np_max_tile( zpic_sim * s, int32_t sp, uint32_t * np ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) );
    unsigned long long st[2]; TRY( np_stats( s, sp, st ) );
    *np = (uint32_t) st[1];
    return ZPIC_OK;
}

static int tiles_host( zpic_sim * s, int sp, std::vector<int> & np, std::vector<int> & poff ) {
    HSpecies * h = s->species[sp];
    np.resize( h->ntiles ); poff.resize( h->ntiles );
    CK( cudaMemcpyAsync( np.data(), h->d.np, h->ntiles * sizeof( int ), cudaMemcpyDeviceToHost, s->stream ) );
    CK( cudaStreamSynchronize( s->stream ) );
    long long o = 0;
    for ( int t = 0; t < h->ntiles; t++ ) { poff[t] = (int) o; o += np[t]; }
    return ZPIC_OK;
}

int zpic_b200_species_get_tiles( zpic_sim * s, int32_t sp, int32_t * np, int32_t * offset ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) );
    std::vector<int> n, o;
    TRY( tiles_host( s, sp, n, o ) );
    if ( np ) std::memcpy( np, n.data(), n.size() * sizeof( int ) );
    if ( offset ) std::memcpy( offset, o.data(), o.size() * sizeof( int ) );
    return ZPIC_OK;
}

int zpic_b200_species_get( zpic_sim * s, int32_t sp, int32_t * ix, float * x, float * u ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) ); TRY( ensure_plan( s ) );
    HSpecies * h = s->species[sp];
    std::vector<int> n, o;
    TRY( tiles_host( s, sp, n, o ) );
    const size_t total = (size_t) o.back() + n.back();
    int * poff_d = nullptr; int2 * ix_d = nullptr; float2 * x_d = nullptr; float * u_d = nullptr;
    TRY( dalloc( &poff_d, h->ntiles ) ); TRY( dalloc( &ix_d, total ) ); TRY( dalloc( &x_d, total ) ); TRY( dalloc( &u_d, 3 * total ) );
    CK( cudaMemcpyAsync( poff_d, o.data(), o.size() * sizeof( int ), cudaMemcpyHostToDevice, s->stream ) );
    CK( launch_pack( s->stream, sp, h->ntiles, s->plan.sps_d, poff_d, ix_d, x_d, u_d ) );
    s->launches++;
    if ( total ) {
        CK( cudaMemcpyAsync( ix, ix_d, total * sizeof( int2 ), cudaMemcpyDeviceToHost, s->stream ) );
        CK( cudaMemcpyAsync( x, x_d, total * sizeof( float2 ), cudaMemcpyDeviceToHost, s->stream ) );
        CK( cudaMemcpyAsync( u, u_d, 3 * total * sizeof( float ), cudaMemcpyDeviceToHost, s->stream ) );
    }
    CK( cudaStreamSynchronize( s->stream ) );
    dfree( poff_d ); dfree( ix_d ); dfree( x_d ); dfree( u_d );
    return check_status( s );
}

int zpic_b200_species_set( zpic_sim * s, int32_t sp, const int32_t * np, const int32_t * ix, const float * x, const float * u ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) );
    HSpecies * h = s->species[sp];
    std::vector<int> n( np, np + h->ntiles );
    uint64_t need = 0;
    for ( int v : n ) {
        if ( v < 0 ) return fail( ZPIC_E_INVALID, "negative particle count" );
        need += roundup4( v );
    }
    CK( cudaStreamSynchronize( s->stream ) );
    // a set larger than the buffer grows it (with a fifth to spare)
    if ( need + 4ull * h->ntiles > h->max_part ) TRY( species_grow( s, h, ( need + 4ull * h->ntiles ) * 6 / 5 ) );
    TRY( species_upload( s, h, n, ix, x, u ) );
    return ZPIC_OK;
}

int zpic_b200_species_gather( zpic_sim * s, int32_t sp, int32_t quant, float * out ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) ); TRY( ensure_plan( s ) );
    if ( quant < 0 || quant > 4 ) return fail( ZPIC_E_INVALID, "invalid quantity" );
    HSpecies * h = s->species[sp];
    std::vector<int> n, o;
    TRY( tiles_host( s, sp, n, o ) );
    const size_t total = (size_t) o.back() + n.back();
    int * poff_d = nullptr; float * out_d = nullptr;
    TRY( dalloc( &poff_d, h->ntiles ) ); TRY( dalloc( &out_d, total ) );
    CK( cudaMemcpyAsync( poff_d, o.data(), o.size() * sizeof( int ), cudaMemcpyHostToDevice, s->stream ) );
    // Species::gather scales positions by dx (species.h:510-526)
    const int scaled = quant <= 1;
    const float sx = quant == 0 ? h->dx[0] : h->dx[1];
    CK( launch_gather( s->stream, sp, h->ntiles, s->plan.sps_d, s->plan.runs_d, poff_d, quant, sx, 0.f, scaled, out_d ) );
    s->launches++;
    if ( total ) CK( cudaMemcpyAsync( out, out_d, total * sizeof( float ), cudaMemcpyDeviceToHost, s->stream ) );
    CK( cudaStreamSynchronize( s->stream ) );
    dfree( poff_d ); dfree( out_d );
    return ZPIC_OK;
}

int zpic_b200_species_charge( zpic_sim * s, int32_t sp, float * out ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) ); TRY( ensure_plan( s ) );
    HSpecies * h = s->species[sp];
    if ( h->sort_pending ) return fail( ZPIC_E_INVALID, "particles have moved since the last tile sort" );
    const int cextx = s->nxx + 1, cexty = s->nxy + 1;
    const int cvol = roundup4( cextx * cexty );
    const size_t nraw = (size_t) cvol * h->ntiles;
    const size_t ndense = (size_t) s->ntx * s->nxx * s->nty * s->nxy;
    float * raw = nullptr; float * dense = nullptr;
    TRY( dalloc( &raw, nraw ) ); TRY( dalloc( &dense, ndense ) );
    CK( cudaMemsetAsync( raw, 0, nraw * sizeof( float ), s->stream ) );
    CK( launch_dep_charge( s->stream, sp, h->ntiles, s->plan.sps_d, s->plan.runs_d, raw, cextx, cvol ) );
    // the charge grid is a new grid object, hence periodic (grid.h:79)
    CK( launch_charge_finish( s->stream, raw, dense, s->ntx, s->nty, s->nxx, s->nxy, cextx, cvol, 1, 1 ) );
    s->launches += 2;
    CK( cudaMemcpyAsync( out, dense, ndense * sizeof( float ), cudaMemcpyDeviceToHost, s->stream ) );
    CK( cudaStreamSynchronize( s->stream ) );
    dfree( raw ); dfree( dense );
    return ZPIC_OK;
}

// Species::dep_phasespace, 1D (species.cpp:2631-2709) and 2D (2863-3022).
// The reference's normalisation calls C's double fabs() on the float charge,
// so that expression is evaluated in double and rounded once to float; the
// range scaling is FP32.
int zpic_b200_species_phasespace( zpic_sim * s, int32_t sp, int32_t quant0, const float range0[2], int32_t size0,
                                  int32_t quant1, const float range1[2], int32_t size1, float * out ) {
    TRY( sim_select( s ) ); TRY( species_index( s, sp ) ); TRY( ensure_plan( s ) );
    if ( !range0 || !out || quant0 < 0 || quant0 > 4 || size0 <= 0 )
        return fail( ZPIC_E_INVALID, "invalid phasespace quantity, range or size" );
    const bool two = quant1 >= 0;
    if ( two ) {
        if ( !range1 || quant1 > 4 || size1 <= 0 ) return fail( ZPIC_E_INVALID, "invalid phasespace quantity, range or size" );
        if ( quant0 >= quant1 )
            return fail( ZPIC_E_INVALID, "for 2D phasespaces, the 2nd quantity must be indexed higher than the first one" );
    }
    HSpecies * h = s->species[sp];
    if ( h->sort_pending ) return fail( ZPIC_E_INVALID, "particles have moved since the last tile sort" );
    float r0[2] = { range0[0], range0[1] }, r1[2] = { 0, 0 };
    if ( two ) { r1[0] = range1[0]; r1[1] = range1[1]; }
    if ( !( r0[1] != r0[0] ) || ( two && !( r1[1] != r1[0] ) ) ) return fail( ZPIC_E_INVALID, "empty phasespace range" );
    PhaSpec p{};
    p.q0 = quant0; p.q1 = two ? quant1 : -1; p.n0 = size0; p.n1 = two ? size1 : 1;
    const float dxy = h->dx[0] * h->dx[1];
    const double aq = std::fabs( (double) h->q );
    if ( !two ) {
        const unsigned usize = (unsigned) size0;
        p.norm = (float) ( aq * dxy * usize / ( r0[1] - r0[0] ) );
    } else {
        const unsigned u0 = (unsigned) size0, u1 = (unsigned) size1;
        p.norm = (float) ( aq * dxy * ( u0 / ( r0[1] - r0[0] ) ) * ( u1 / ( r1[1] - r1[0] ) ) );
    }
    // positions are deposited in cell units
    for ( int k = 0; k < 2; k++ ) {
        if ( quant0 < 2 ) r0[k] /= h->dx[ quant0 ];
        if ( two && quant1 < 2 ) r1[k] /= h->dx[ quant1 ];
    }
    p.r0 = r0[0]; p.rdx0 = size0 / ( r0[1] - r0[0] );
    if ( two ) { p.r1 = r1[0]; p.rdx1 = size1 / ( r1[1] - r1[0] ); }
    const size_t nbins = (size_t) size0 * ( two ? size1 : 1 );
    float * d = nullptr;
    TRY( dalloc( &d, nbins ) );
    CK( cudaMemsetAsync( d, 0, nbins * sizeof( float ), s->stream ) );
    CK( launch_phasespace( s->stream, sp, h->ntiles, s->plan.sps_d, s->plan.runs_d, p, d ) );
    s->launches += 1;
    CK( cudaMemcpyAsync( out, d, nbins * sizeof( float ), cudaMemcpyDeviceToHost, s->stream ) );
    CK( cudaStreamSynchronize( s->stream ) );
    dfree( d );
    return check_status( s );
}

// ---- grids ----
static float * grid_ptr( zpic_sim * s, int which, bool for_read ) {
    switch ( which ) {
    case ZPIC_GRID_E: return s->run.E;
    case ZPIC_GRID_B: return s->run.B;
    case ZPIC_GRID_J: return ( for_read && !s->j_final ) ? s->run.Jdep : s->run.J;
    }
    return nullptr;
}

int zpic_b200_grid_size( zpic_sim * s, int32_t which, uint64_t * cells ) {
    if ( !s || !cells || which < 0 || which > 2 ) return fail( ZPIC_E_INVALID, "invalid argument" );
    *cells = (uint64_t) s->run.tile_vol * s->ntx * s->nty;
    return ZPIC_OK;
}

int zpic_b200_grid_get( zpic_sim * s, int32_t which, float * out ) {
    TRY( sim_select( s ) );
    float * p = grid_ptr( s, which, true );
    if ( !p || !out ) return fail( ZPIC_E_INVALID, "invalid grid" );
    CK( cudaMemcpyAsync( out, p, s->grid_floats() * sizeof( float ), cudaMemcpyDeviceToHost, s->stream ) );
    CK( cudaStreamSynchronize( s->stream ) );
    return ZPIC_OK;
}

int zpic_b200_grid_set( zpic_sim * s, int32_t which, const float * in ) {
    TRY( sim_select( s ) );
    // J: the buffer grid_get returns (raw deposits before Current::advance, else the summed current)
    float * p = grid_ptr( s, which, true );
    if ( !p || !in ) return fail( ZPIC_E_INVALID, "invalid grid" );
    CK( cudaMemcpyAsync( p, in, s->grid_floats() * sizeof( float ), cudaMemcpyHostToDevice, s->stream ) );
    CK( cudaStreamSynchronize( s->stream ) );
    if ( which == ZPIC_GRID_J && !s->j_final ) s->jdep_clean = false;
    return ZPIC_OK;
}

int zpic_b200_grid_gather( zpic_sim * s, int32_t which, int32_t fc, float * out ) {
    TRY( sim_select( s ) );
    float * p = grid_ptr( s, which, true );
    if ( !p || !out || fc < 0 || fc > 2 ) return fail( ZPIC_E_INVALID, "invalid grid" );
    const size_t n = (size_t) s->ntx * s->nxx * s->nty * s->nxy;
    float * d = nullptr;
    TRY( dalloc( &d, n ) );
    CK( launch_grid_gather( s->stream, p, d, fc, s->ntx, s->nty, s->nxx, s->nxy, s->run.extx, s->run.gc_off, s->run.tile_vol ) );
    s->launches++;
    CK( cudaMemcpyAsync( out, d, n * sizeof( float ), cudaMemcpyDeviceToHost, s->stream ) );
    CK( cudaStreamSynchronize( s->stream ) );
    dfree( d );
    return ZPIC_OK;
}

// ---- batches ----
int zpic_b200_batch_create( zpic_sim * const * sims, int32_t n, zpic_batch ** out ) {
    if ( !sims || n <= 0 || !out ) return fail( ZPIC_E_INVALID, "invalid batch" );
    auto b = std::make_unique<zpic_batch>();
    for ( int i = 0; i < n; i++ ) {
        if ( !sims[i] ) return fail( ZPIC_E_INVALID, "null simulation in batch" );
        if ( sims[i]->device != sims[0]->device ) return fail( ZPIC_E_INVALID, "batch simulations must share a device" );
        if ( sims[i]->emf_mw.active ) return fail( ZPIC_E_INVALID, "moving-window simulations cannot be batched" );
        b->sims.push_back( sims[i] );
    }
    CK( cudaSetDevice( sims[0]->device ) );
    CK( cudaStreamCreateWithFlags( &b->stream, cudaStreamNonBlocking ) );
    CK( cudaEventCreateWithFlags( &b->ev, cudaEventDisableTiming ) );
    TRY( plan_build( b->plan, b->sims, b->chunks ) );
    for ( auto * s : b->sims ) b->gens.push_back( s->layout_gen );
    *out = b.release();
    return ZPIC_OK;
}

// A run whose buffers or descriptors changed since the batch's plan was built
// (options, boundaries, particle-buffer growth) makes the batch rebuild it.
static int batch_refresh( zpic_batch * b ) {
    bool stale = b->gens.size() != b->sims.size();
    for ( size_t i = 0; i < b->sims.size() && !stale; i++ ) stale = b->gens[i] != b->sims[i]->layout_gen;
    if ( !stale ) return ZPIC_OK;
    for ( auto * s : b->sims ) CK( cudaStreamSynchronize( s->stream ) );
    CK( cudaStreamSynchronize( b->stream ) );
    TRY( plan_build( b->plan, b->sims, b->chunks ) );
    b->gens.clear();
    for ( auto * s : b->sims ) b->gens.push_back( s->layout_gen );
    return ZPIC_OK;
}

int zpic_b200_batch_advance( zpic_batch * b, int32_t nsteps ) {
    if ( !b ) return fail( ZPIC_E_INVALID, "null batch" );
    CK( cudaSetDevice( b->sims[0]->device ) );
    TRY( batch_refresh( b ) );
    for ( auto * s : b->sims ) {
        if ( !s->plan.built ) TRY( ensure_plan( s ) );
        CK( cudaEventRecord( b->ev, s->stream ) );
        CK( cudaStreamWaitEvent( b->stream, b->ev, 0 ) );
        for ( auto * sp : s->species )
            if ( sp->counters_dirty ) {
                CK( cudaMemsetAsync( sp->d.cnt, 0, 9 * (size_t) sp->ntiles * sizeof( int ), b->stream ) );
                CK( cudaMemsetAsync( sp->d.nidx, 0, sp->ntiles * sizeof( int ), b->stream ) );
                sp->counters_dirty = false;
            }
    }
    uint64_t l = 0;
    TRY( plan_advance( b->plan, b->stream, nsteps, true, &l ) );
    b->launches += l;
    CK( cudaEventRecord( b->ev, b->stream ) );
    for ( auto * s : b->sims ) CK( cudaStreamWaitEvent( s->stream, b->ev, 0 ) );
    return ZPIC_OK;
}

int zpic_b200_sim_autotune( zpic_sim * s, int32_t steps, int32_t * chosen ) {
    TRY( sim_select( s ) );
    if ( steps < 1 ) return fail( ZPIC_E_INVALID, "autotune needs at least one timed step" );
    if ( s->species.empty() ) return fail( ZPIC_E_INVALID, "no species to tune for" );
    if ( s->emf_mw.active ) return fail( ZPIC_E_INVALID, "autotune runs Simulation::advance steps; not for moving-window runs" );
    uint64_t ntiles = 0; for ( auto * h : s->species ) ntiles += h->ntiles;
    const int automatic = auto_chunks( (int) ntiles, 0 );
    int best = automatic; float best_ms = -1;
    for ( int c : chunk_candidates( particles_of( s ), ntiles, automatic ) ) {
        TRY( zpic_b200_sim_set_option( s, "chunks", c ) );
        float ms = 0;
        TRY( time_candidate( s->stream, steps, [&]( int n ) { return zpic_b200_sim_advance( s, n ); }, &ms ) );
        if ( best_ms < 0 || ms < best_ms ) { best_ms = ms; best = c; }
    }
    TRY( zpic_b200_sim_set_option( s, "chunks", best ) );
    if ( chosen ) *chosen = best;
    return ZPIC_OK;
}

int zpic_b200_batch_autotune( zpic_batch * b, int32_t steps, int32_t * chosen ) {
    if ( !b ) return fail( ZPIC_E_INVALID, "null batch" );
    if ( steps < 1 ) return fail( ZPIC_E_INVALID, "autotune needs at least one timed step" );
    CK( cudaSetDevice( b->sims[0]->device ) );
    uint64_t ntiles = 0, np = 0;
    for ( auto * s : b->sims ) { np += particles_of( s ); for ( auto * h : s->species ) ntiles += h->ntiles; }
    const int automatic = auto_chunks( (int) std::min<uint64_t>( ntiles, 1u << 30 ), 0 );
    int best = automatic; float best_ms = -1;
    for ( int c : chunk_candidates( np, ntiles, automatic ) ) {
        if ( c < 0 ) continue;          // a batch chunks all of its runs alike
        b->chunks = c;
        TRY( plan_build( b->plan, b->sims, c ) );
        float ms = 0;
        TRY( time_candidate( b->stream, steps, [&]( int n ) { return zpic_b200_batch_advance( b, n ); }, &ms ) );
        if ( best_ms < 0 || ms < best_ms ) { best_ms = ms; best = c; }
    }
    b->chunks = best;
    TRY( plan_build( b->plan, b->sims, best ) );
    if ( chosen ) *chosen = best;
    return ZPIC_OK;
}

int zpic_b200_batch_launch_count( zpic_batch * b, uint64_t * count ) {
    if ( !b || !count ) return fail( ZPIC_E_INVALID, "null argument" );
    *count = b->launches;
    return ZPIC_OK;
}

int zpic_b200_batch_stream( zpic_batch * b, void ** stream ) {
    if ( !b || !stream ) return fail( ZPIC_E_INVALID, "null argument" );
    *stream = (void *) b->stream;
    return ZPIC_OK;
}

int zpic_b200_batch_synchronize( zpic_batch * b ) {
    if ( !b ) return fail( ZPIC_E_INVALID, "null batch" );
    CK( cudaSetDevice( b->sims[0]->device ) );
    CK( cudaStreamSynchronize( b->stream ) );
    for ( auto * s : b->sims ) TRY( check_status( s ) );
    return ZPIC_OK;
}

int zpic_b200_batch_destroy( zpic_batch * b ) {
    if ( !b ) return ZPIC_OK;
    cudaSetDevice( b->sims[0]->device );
    cudaStreamSynchronize( b->stream );
    b->plan.release();
    cudaEventDestroy( b->ev );
    cudaStreamDestroy( b->stream );
    delete b;
    return ZPIC_OK;
}

}  // extern "C"
