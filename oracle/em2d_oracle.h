/*
 * em2d_oracle.h -- plain-C restatement of the zpic-parallel openmp/em2d time
 * step (push, move + charge-conserving deposit, particle boundary conditions,
 * tile sort, current guard cells / filter, Yee solver, moving window,
 * initial conditions and lasers).
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker the CUDA path is compared
 * against.  It is never linked into, loaded by or called from the product.
 *
 * Built twice by oracle/Makefile: ORACLE_REAL=float (bit-exact restatement
 * of the reference's scalar FP32 build, pinned against oracle/_ref) and
 * ORACLE_REAL=double (the FP64 build of the same path).
 *
 * Layouts follow the reference:
 *   grids  -- per-tile blocks of tile_vol = roundup4(ext_x*ext_y) cells,
 *             guard cells {1,2} per axis for E, B, J (grid.h:77-92)
 *   particles -- packed per tile at offset[t]: ix (2 ints), x (2 reals),
 *             u (3 reals) per particle (particles.h:82-105)
 */
#ifndef EM2D_ORACLE_H_
#define EM2D_ORACLE_H_

#include <stdint.h>

#ifndef ORACLE_REAL
#define ORACLE_REAL float
#endif
typedef ORACLE_REAL real;

typedef struct osim osim;

/* density types: 0 None, 1 Uniform, 2 Step, 3 Slab, 4 Sphere; p = {n0, a, b, c, dir} */
/* udist types: 0 None, 1 Cold, 2 Thermal, 3 ThermalCorr */
/* bc arrays: {x.lower, x.upper, y.lower, y.upper} */

int      oracle_real_size( void );
osim *   osim_create( unsigned ntx, unsigned nty, unsigned nxx, unsigned nxy,
                      float boxx, float boxy, double dt );
void     osim_destroy( osim * s );
int      osim_add_species( osim * s, float m_q, unsigned ppcx, unsigned ppcy,
                           int dens_type, const float * dens_p,
                           int udist_type, const float * uth, const float * ufl, int npmin,
                           int push_type, const int * bc );
void     osim_set_moving_window( osim * s );
void     osim_emf_set_bc( osim * s, const int * bc );
void     osim_current_set_bc( osim * s, const int * bc );
void     osim_current_set_filter( osim * s, int type, int dir, unsigned order );
int      osim_add_laser( osim * s, int type, const float * p );

void     osim_advance( osim * s, int n );
void     osim_advance_mov_window( osim * s, int n );
void     osim_current_zero( osim * s );
void     osim_current_advance( osim * s );
void     osim_emf_advance( osim * s, int with_current );
void     osim_species_advance( osim * s, int sp );
void     osim_species_advance_free( osim * s, int sp );
void     osim_species_push( osim * s, int sp );
void     osim_species_move( osim * s, int sp );
void     osim_species_process_bc( osim * s, int sp );
void     osim_species_tile_sort( osim * s, int sp );

void     osim_set_clock( osim * s, unsigned k );
unsigned osim_iter( osim * s );
uint64_t osim_nmove( osim * s );
double   osim_species_energy( osim * s, int sp );
void     osim_emf_energy( osim * s, double * out6 );
uint64_t osim_species_tiles( osim * s, int sp, int * np, int * offset );
uint32_t osim_species_max_part( osim * s, int sp );
void     osim_species_get( osim * s, int sp, int * ix, real * x, real * u );
int      osim_species_set( osim * s, int sp, const int * np, const int * ix, const real * x, const real * u );
uint64_t osim_grid_size( osim * s, int which );
void     osim_grid_get( osim * s, int which, real * out );
void     osim_grid_set( osim * s, int which, const real * in );
void     osim_species_charge( osim * s, int sp, real * out );
int      osim_species_phasespace( osim * s, int sp, int q0, const float * range0, int size0,
                                  int q1, const float * range1, int size1, real * out );

#endif
