/*
 * zpic_b200.h -- C-ABI of libzpic_b200.so, the B200 (sm_100a) em2d time step.
 *
 * Every entry point is `extern "C"`, takes plain pointers, sizes and
 * fixed-width integers, and returns an int status: 0 on success, a negative
 * ZPIC_E_* code on error (zpic_b200_last_error() then returns a message).
 * Host buffers belong to the caller; device buffers belong to the library.
 *
 * Each group of entry points names the reference interface it replaces
 * (paths relative to the zpic-parallel project, openmp/em2d/).  The C++
 * drop-in classes in zpic-parallel_b200/cpp/ (Simulation, Species, EMF,
 * Current, ...) are thin wrappers over these calls.
 *
 * Threading: one host thread per simulation handle; calls on one handle are
 * not re-entrant (as in the reference, simulation.h).  Calls that return
 * data to the host synchronise the handle's CUDA stream.
 */
#ifndef ZPIC_B200_H_
#define ZPIC_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define ZPIC_OK              0
#define ZPIC_E_INVALID      -1   /* invalid argument / parameter */
#define ZPIC_E_CUDA         -2   /* CUDA runtime error */
#define ZPIC_E_NOMEM        -3   /* allocation failed / particle buffer overflow */
#define ZPIC_E_STATE        -4   /* call not allowed in the current state */
#define ZPIC_E_DEVICE       -5   /* a kernel reported an error (bounded wait expired, capacity) */

/* ---- enums (values match the reference's enums) ---- */
/* species::bc (species.h:43-47) */
#define ZPIC_SPECIES_BC_OPEN        0
#define ZPIC_SPECIES_BC_PERIODIC    1
#define ZPIC_SPECIES_BC_REFLECTING  2
/* emf::bc (emf.h:16-22) */
#define ZPIC_EMF_BC_NONE     0
#define ZPIC_EMF_BC_PERIODIC 1
#define ZPIC_EMF_BC_PEC      2
#define ZPIC_EMF_BC_PMC      3
/* current::bc (current.h:10-15) */
#define ZPIC_CURRENT_BC_NONE       0
#define ZPIC_CURRENT_BC_PERIODIC   1
#define ZPIC_CURRENT_BC_REFLECTING 2
/* species::pusher (species.h:43) */
#define ZPIC_PUSH_BORIS 0
#define ZPIC_PUSH_EULER 1
/* Density::* (density.h:12-131) */
#define ZPIC_DENSITY_NONE    0
#define ZPIC_DENSITY_UNIFORM 1
#define ZPIC_DENSITY_STEP    2
#define ZPIC_DENSITY_SLAB    3
#define ZPIC_DENSITY_SPHERE  4
/* UDistribution::* (udist.h:11-58) */
#define ZPIC_UDIST_NONE        0
#define ZPIC_UDIST_COLD        1
#define ZPIC_UDIST_THERMAL     2
#define ZPIC_UDIST_THERMALCORR 3
/* Filter::* (filter.h:9-86) */
#define ZPIC_FILTER_NONE        0
#define ZPIC_FILTER_BINOMIAL    1
#define ZPIC_FILTER_COMPENSATED 2
/* Laser::* (laser.h:8-131) */
#define ZPIC_LASER_PLANE    0
#define ZPIC_LASER_GAUSSIAN 1
/* grids */
#define ZPIC_GRID_E 0
#define ZPIC_GRID_B 1
#define ZPIC_GRID_J 2
/* part::quant (particles.h:16-18) */
#define ZPIC_QUANT_X  0
#define ZPIC_QUANT_Y  1
#define ZPIC_QUANT_UX 2
#define ZPIC_QUANT_UY 3
#define ZPIC_QUANT_UZ 4
/* Species advance modes */
#define ZPIC_ADVANCE_FULL    0   /* Species::advance(EMF const&, Current&)  species.cpp:2051 */
#define ZPIC_ADVANCE_CURRENT 1   /* Species::advance(Current&)              species.cpp:2025 */
#define ZPIC_ADVANCE_FREE    2   /* Species::advance()                      species.cpp:1998 */

typedef struct zpic_sim   zpic_sim;    /* one Simulation (EMF + Current + species) */
typedef struct zpic_batch zpic_batch;  /* several Simulations stepped together      */

/* Density::Profile (density.h:12-131): a,b,c = step pos | slab begin,end | sphere cx,cy,r */
typedef struct {
    int32_t type;
    float   n0;
    float   a, b, c;
    int32_t dir;       /* coord::cart: 0 x, 1 y */
} zpic_density;

/* UDistribution::Type (udist.h:11-58) */
typedef struct {
    int32_t type;
    float   uth[3];
    float   ufl[3];
    int32_t npmin;     /* ThermalCorr only (default 2) */
} zpic_udist;

/* Species( name, m_q, ppc ) + set_density / set_udist / set_bc / push_type
 * (species.h:147-265, species.cpp:1693-1718) */
typedef struct {
    const char * name;
    float        m_q;
    uint32_t     ppc[2];
    zpic_density density;
    zpic_udist   udist;
    int32_t      push_type;
    int32_t      bc[4];          /* {x.lower, x.upper, y.lower, y.upper} */
} zpic_species_desc;

/* Laser::PlaneWave / Laser::Gaussian public fields (laser.h:8-131) */
typedef struct {
    int32_t type;
    float start, fwhm, rise, flat, fall;
    float a0, omega0, polarization, cos_pol, sin_pol;
    uint32_t filter;             /* default 1 */
    float W0, focus, axis;       /* Gaussian only */
} zpic_laser_desc;

/* ---- library ---- */
const char * zpic_b200_last_error( void );
int zpic_b200_version( void );
/* Selects the CUDA device used by simulations created afterwards on this host thread. */
int zpic_b200_set_device( int device );

/* ---- Simulation (simulation.h:39-180) ---- */
/* Simulation( ntiles, nx, box, dt ): builds EMF (emf.cpp:16-54, Courant check) and Current (current.cpp:14-42) */
int zpic_b200_sim_create( uint32_t ntiles_x, uint32_t ntiles_y, uint32_t nx_x, uint32_t nx_y,
                          float box_x, float box_y, double dt, zpic_sim ** out );
int zpic_b200_sim_destroy( zpic_sim * sim );
/* Simulation::add_species (simulation.h:68-71) -> Species::initialize (species.cpp:1730-1788) */
int zpic_b200_sim_add_species( zpic_sim * sim, const zpic_species_desc * desc, int32_t * species_id );
/* Simulation::set_moving_window (simulation.h:56-62) */
int zpic_b200_sim_set_moving_window( zpic_sim * sim );
/* Simulation::advance / advance_mov_window, nsteps times (simulation.h:90-130) */
int zpic_b200_sim_advance( zpic_sim * sim, int32_t nsteps );
int zpic_b200_sim_advance_mov_window( zpic_sim * sim, int32_t nsteps );
/* Simulation::get_iter / get_nmove (simulation.h:136-180) */
int zpic_b200_sim_iter( zpic_sim * sim, uint32_t * iter );
int zpic_b200_sim_nmove( zpic_sim * sim, uint64_t * nmove );
int zpic_b200_sim_synchronize( zpic_sim * sim );
/*
 * Tuning / instrumentation knobs (no reference counterpart):
 *   "graph"          1/0  capture repeated steps in a CUDA graph (default 1)
 *   "chunks"         n    CTAs per tile in the particle kernel: n > 0 for every
 *                         tile, 0 automatic (default), -1 automatic and in
 *                         proportion to each tile's particles
 *   "profile"        0/1/2 phase timing read by zpic_b200_sim_phase_times: 1
 *                         CUDA events around each kernel phase, steps issued
 *                         without a graph; 2 events around the particle kernel
 *                         as nodes of the step graph (graph replays timed)
 *   "jacc"           0/1/2 tile current accumulation in shared memory: 0 FP32
 *                         atomics (the reference's FP32 sums, in another order),
 *                         1 FP64 atomics, 2 fixed point (default: the FP32
 *                         contributions rounded to 2^-29 |q| and summed exactly
 *                         in integer arithmetic, independent of the order of
 *                         the additions; the fastest of the three)
 *   "reorder"        n    every n steps, put each tile's particles back into
 *                         cell round-robin order (one particle of every cell,
 *                         cells ascending, then the next round), which keeps
 *                         the particle kernel's shared-memory bank conflicts at
 *                         their initial level; 0 never.  Default: every 50
 *                         steps, never in a moving-window run.  Order only:
 *                         every tile keeps its particle multiset.
 *   "capacity_factor" f   initial particle capacity of species added after
 *                         this call: f * cells * ppc (default 1.6; the
 *                         reference's max_part is 1.2 * cells * ppc,
 *                         species.cpp:1752, for a layout without per-tile
 *                         room); buffers grow when injection or species_set
 *                         needs more
 *   "pool_fraction"  f    share of the free particle capacity kept as a pool
 *                         after the last tile slot (default 0.25); a tile whose
 *                         particles outgrow its slot moves into the pool, and
 *                         only when the pool is short is the whole layout
 *                         rebuilt.  Set before adding species to affect their
 *                         first layout.  Order only: results do not change
 *   "relocation_room" r   room a moved tile gets beyond its particles, as a
 *                         share of their number (default 0.5; at least twice
 *                         the minimum slack of ppc * cells / 8)
 *   "wait_limit"     n    polls before a kernel's bounded wait on its bulk
 *                         copies gives up (default 4194304, ~0.5 s); a kernel
 *                         that gives up skips its work for that tile and the
 *                         next synchronising call returns ZPIC_E_DEVICE
 */
int zpic_b200_sim_set_option( zpic_sim * sim, const char * key, double value );
/* Autotuner (no reference counterpart): times `steps` steps for each
 * candidate number of CTAs per tile -- the "chunks" values 0 and -1
 * (automatic; -1 in proportion to each tile's particles) and 1, 2, 4, ... 64
 * (at least 256 particles per CTA on average) -- and keeps the fastest;
 * *chosen gets it.  The trial steps are real Simulation::advance steps (each candidate
 * runs 1 + steps of them); the choice changes no result beyond the FP32
 * order in which per-CTA partial currents are added.  Not for moving-window
 * simulations. */
int zpic_b200_sim_autotune( zpic_sim * sim, int32_t steps, int32_t * chosen );
/* Per-phase device time (ms) and launch counts accumulated while "profile" is on.
 * phases: 0 particle kernel, 1 sort, 2 current, 3 field solve, 4 other.  n <= 5. */
int zpic_b200_sim_phase_times( zpic_sim * sim, double * ms, uint64_t * launches, int32_t n );
int zpic_b200_sim_reset_phase_times( zpic_sim * sim );
/* Kernel launches issued by the library for this handle since creation. */
int zpic_b200_sim_launch_count( zpic_sim * sim, uint64_t * count );
/* The cudaStream_t of this handle (for external event timing).  Every call's
 * work is ordered on it: a step also runs part of its kernels on a second,
 * internal stream, forked from this one and joined back into it before the
 * step ends, so events recorded on it bracket whole calls. */
int zpic_b200_sim_stream( zpic_sim * sim, void ** stream );

/* ---- EMF (emf.h:24-197) ---- */
int zpic_b200_emf_set_bc( zpic_sim * sim, const int32_t bc[4] );          /* EMF::set_bc */
int zpic_b200_emf_advance( zpic_sim * sim, int32_t with_current );        /* EMF::advance() / advance(Current&) */
int zpic_b200_emf_energy( zpic_sim * sim, double ene_E[3], double ene_B[3] ); /* EMF::get_energy (emf.cpp:662) */
int zpic_b200_laser_add( zpic_sim * sim, const zpic_laser_desc * laser ); /* Laser::Pulse::add (laser.h:85-99) */

/* ---- Current (current.h:17-148) ---- */
int zpic_b200_current_set_bc( zpic_sim * sim, const int32_t bc[4] );      /* Current::set_bc */
int zpic_b200_current_set_filter( zpic_sim * sim, int32_t type, int32_t dir, uint32_t order ); /* Current::set_filter */
int zpic_b200_current_zero( zpic_sim * sim );                             /* Current::zero (current.cpp:253) */
int zpic_b200_current_advance( zpic_sim * sim );                          /* Current::advance (current.cpp:227) */

/* ---- Species (species.h:147-528) ---- */
int zpic_b200_species_advance( zpic_sim * sim, int32_t sp, int32_t mode );     /* Species::advance overloads */
int zpic_b200_species_advance_mov_window( zpic_sim * sim, int32_t sp );        /* species.cpp:2083-2128 */
int zpic_b200_species_push( zpic_sim * sim, int32_t sp );                      /* Species::push (species.cpp:2302) */
int zpic_b200_species_move( zpic_sim * sim, int32_t sp );                      /* Species::move(J) (species.cpp:2138) */
int zpic_b200_species_process_bc( zpic_sim * sim, int32_t sp );                /* Species::process_bc (species.cpp:1967) */
int zpic_b200_species_tile_sort( zpic_sim * sim, int32_t sp );                 /* Particles::tile_sort (particles.cpp:855) */
int zpic_b200_species_set_bc( zpic_sim * sim, int32_t sp, const int32_t bc[4] ); /* Species::set_bc (species.h:211) */
int zpic_b200_species_set_push_type( zpic_sim * sim, int32_t sp, int32_t type );
int zpic_b200_species_energy( zpic_sim * sim, int32_t sp, double * energy );   /* Species::get_energy (species.h:365) */
int zpic_b200_species_nmove( zpic_sim * sim, int32_t sp, uint64_t * nmove );   /* Species::get_nmove */
int zpic_b200_species_np_total( zpic_sim * sim, int32_t sp, uint64_t * np );   /* Species::np_total */
/* Times the tile sort had to rebuild the slot layout of this species (a full
 * copy of its particles through the second buffer); no reference counterpart. */
int zpic_b200_species_repacks( zpic_sim * sim, int32_t sp, uint64_t * repacks );
/* Tiles that outgrew their slot and were moved into the free pool at the
 * end of the buffer (instead of a repack); no reference counterpart. */
int zpic_b200_species_relocations( zpic_sim * sim, int32_t sp, uint64_t * tiles );
int zpic_b200_species_np_max_tile( zpic_sim * sim, int32_t sp, uint32_t * np );/* Species::np_max_tile */
/* Particle-buffer capacity (the public Particles::max_part, particles.h:82-105).
 * It grows, as the reference's does in its sort (particles.cpp:863-888), when
 * injection or species_set needs more room. */
int zpic_b200_species_max_part( zpic_sim * sim, int32_t sp, uint32_t * max_part );
/* Tile information in the reference's packed layout: offset[t] = sum of np before t (particles.h:94-97) */
int zpic_b200_species_get_tiles( zpic_sim * sim, int32_t sp, int32_t * np, int32_t * offset );
/* Particle data in the reference's packed layout (ix: 2 int32, x: 2 float, u: 3 float per particle) */
int zpic_b200_species_get( zpic_sim * sim, int32_t sp, int32_t * ix, float * x, float * u );
int zpic_b200_species_set( zpic_sim * sim, int32_t sp, const int32_t * np,
                           const int32_t * ix, const float * x, const float * u );
/* Species::gather (species.h:510-526): positions in simulation units, packed tile order */
int zpic_b200_species_gather( zpic_sim * sim, int32_t sp, int32_t quant, float * out );
/* Species::deposit_charge + add_from_gc as save_charge builds it (species.cpp:2486-2511); dense [ny][nx] */
int zpic_b200_species_charge( zpic_sim * sim, int32_t sp, float * out );
/* Species::dep_phasespace (species.cpp:2631-2709 1D, 2863-3022 2D): phase-space
 * density of a species into out[size0] (quant1 < 0) or out[size1][size0].
 * Quantities: ZPIC_PHA_X, _Y (positions, range in simulation units), _UX, _UY,
 * _UZ.  A 2D phase space needs quant1 > quant0 (the reference's rule).  The
 * bins are FP32 sums like the reference's; their order of summation differs. */
enum { ZPIC_PHA_X = 0, ZPIC_PHA_Y = 1, ZPIC_PHA_UX = 2, ZPIC_PHA_UY = 3, ZPIC_PHA_UZ = 4 };
int zpic_b200_species_phasespace( zpic_sim * sim, int32_t sp, int32_t quant0, const float range0[2], int32_t size0,
                                  int32_t quant1, const float range1[2], int32_t size1, float * out );

/* ---- grids (grid.h / vec3grid.h) ---- */
/* cells in the tiled buffer, guard cells and padding included: ntiles * tile_vol */
int zpic_b200_grid_size( zpic_sim * sim, int32_t which, uint64_t * cells );
/* tiled float3 buffer (the reference's d_buffer layout, grid.h:77-92) */
int zpic_b200_grid_get( zpic_sim * sim, int32_t which, float * out );
int zpic_b200_grid_set( zpic_sim * sim, int32_t which, const float * in );
/* vec3grid::gather (vec3grid.h:76-205): one component, dense [ny][nx] */
int zpic_b200_grid_gather( zpic_sim * sim, int32_t which, int32_t fc, float * out );

/*
 * ---- charge density without device allocation ----
 * No counterpart in the reference.  Same result as zpic_b200_species_charge
 * (dense [ny][nx] charge density of one particle set), for callers that
 * cannot allocate device memory: a host framework that owns all device
 * memory through its own pool and forbids foreign allocations, or a
 * real-time or in-situ analysis loop inside another code's time step that
 * must not stall on the allocator (cudaMalloc may synchronise the device).
 * The caller passes device pointers: per-tile particle counts and offsets of
 * a packed particle set (the layout zpic_b200_species_get returns: ix as
 * 2 int32, x as 2 float per particle), the charge per particle q, and the
 * output grid of ntiles_x*nx_x * ntiles_y*nx_y floats; work is queued on
 * `stream` (a cudaStream_t, or NULL for the default stream).
 * Precondition: every particle's cell lies inside its tile,
 * 0 <= ix.x < nx_x and 0 <= ix.y < nx_y (a sorted set, as species_get returns
 * it); particles outside are skipped, not deposited.
 * Scratch lives in a fixed 32 MiB device array owned by the library (held on
 * every GPU that loads it until exit).  Limits, checked before any work is
 * queued (ZPIC_E_INVALID otherwise): a tile block of (nx_x+1)*(nx_y+1) cells
 * at most 12288, and ntiles_x*ntiles_y * roundup4((nx_x+1)*(nx_y+1)) at most
 * 8 Mi floats.  The first call on a device (and the first after that
 * device's context was reset) resolves the array's address on that device
 * with a host-side lookup.  All calls share the
 * array, which keeps the last call's contents (each call clears the part it
 * uses): calls that overlap on the GPU race and must be serialised.
 */
int zpic_b200_charge_deposit_noalloc( uint32_t ntiles_x, uint32_t ntiles_y, uint32_t nx_x, uint32_t nx_y,
                                      float q, const int32_t * np, const int32_t * offset,
                                      const int32_t * ix, const float * x, float * charge, void * stream );

/* ---- batched ensembles (no reference counterpart: many independent runs per launch) ---- */
int zpic_b200_batch_create( zpic_sim * const * sims, int32_t n, zpic_batch ** out );
int zpic_b200_batch_advance( zpic_batch * batch, int32_t nsteps );
int zpic_b200_batch_synchronize( zpic_batch * batch );
int zpic_b200_batch_destroy( zpic_batch * batch );
/* The autotuner above for a batch: CTAs per tile for all of its runs. */
int zpic_b200_batch_autotune( zpic_batch * batch, int32_t steps, int32_t * chosen );
/* Kernel launches issued by batch steps since the batch was created. */
int zpic_b200_batch_launch_count( zpic_batch * batch, uint64_t * count );
/* The cudaStream_t a batch's steps run on (for external event timing). */
int zpic_b200_batch_stream( zpic_batch * batch, void ** stream );

#ifdef __cplusplus
}
#endif

#endif
