/*
 * ref_harness.cpp -- ctypes-callable harness around the UNMODIFIED reference
 * OpenMP em2d sources (zpic-parallel, openmp/em2d/).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is compiled together with the
 * reference's own .cpp files by oracle/Makefile into oracle/_ref/.  Only the
 * tests, __graft_entry__.smoke() and bench.py's reference / cpu_baseline arms
 * may load the resulting library; the product never does.
 *
 * It drives the reference's public C++ API exactly as its test drivers do
 * (openmp/em2d/main.cpp:179-259 test_weibel, 540-607 test_lwfa) and exposes
 * the state through plain C entry points so the Python tests can pin the
 * plain-C restatement (oracle/em2d_oracle.c) and the CUDA path against it.
 *
 * Reference-side quirks handled here (see openmp/em2d sources):
 *   - Species::particles is protected (species.h:83), so a thin subclass
 *     exposes it.
 *   - Species::save() crashes under libstdc++ (species.cpp:2421-2450 casts
 *     std::string[] to char**); it is never called.
 */
#include "simulation.h"
#include "laser.h"
#include "filter.h"
#include "density.h"
#include "udist.h"

#include <vector>
#include <cstring>
#include <cstdint>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

class HSpecies : public Species {
public:
    HSpecies( std::string const name, float const m_q, uint2 const ppc ) : Species( name, m_q, ppc ) {}
    Particles * parts() { return particles; }
    Particles * tmp_parts() { return tmp; }
    ParticleSort * sorter() { return sort; }
    void bc() { process_bc(); }
};

struct RefSim {
    Simulation * sim;
    std::vector<HSpecies *> species;
};

Density::Profile * make_density( int type, const float * p ) {
    // p = { n0, a, b, c, dir }
    coord::cart dir = ( p && p[4] != 0 ) ? coord::y : coord::x;
    switch ( type ) {
    case 0: return new Density::None();
    case 1: return new Density::Uniform( p[0] );
    case 2: return new Density::Step( dir, p[0], p[1] );
    case 3: return new Density::Slab( dir, p[0], p[1], p[2] );
    case 4: return new Density::Sphere( p[0], make_float2( p[1], p[2] ), p[3] );
    }
    return nullptr;
}

UDistribution::Type * make_udist( int type, const float * uth, const float * ufl, int npmin ) {
    switch ( type ) {
    case 0: return new UDistribution::None();
    case 1: return new UDistribution::Cold( make_float3( ufl[0], ufl[1], ufl[2] ) );
    case 2: return new UDistribution::Thermal( make_float3( uth[0], uth[1], uth[2] ),
                                               make_float3( ufl[0], ufl[1], ufl[2] ) );
    case 3: return new UDistribution::ThermalCorr( make_float3( uth[0], uth[1], uth[2] ),
                                                   make_float3( ufl[0], ufl[1], ufl[2] ), npmin );
    }
    return nullptr;
}

vec3grid<float3> * pick_grid( RefSim * s, int which ) {
    switch ( which ) {
    case 0: return s->sim->emf.E;
    case 1: return s->sim->emf.B;
    case 2: return s->sim->current.J;
    }
    return nullptr;
}

}

extern "C" {

int ref_num_threads( int n ) {
#ifdef _OPENMP
    if ( n > 0 ) omp_set_num_threads( n );
    return omp_get_max_threads();
#else
    (void) n;
    return 1;
#endif
}

void * ref_sim_create( unsigned ntx, unsigned nty, unsigned nxx, unsigned nxy,
                       float boxx, float boxy, double dt ) {
    RefSim * s = new RefSim;
    s->sim = new Simulation( make_uint2( ntx, nty ), make_uint2( nxx, nxy ),
                             make_float2( boxx, boxy ), dt );
    return s;
}

void ref_sim_destroy( void * h ) {
    RefSim * s = static_cast<RefSim *>( h );
    delete s->sim;          // Simulation holds non-owning Species pointers
    for ( auto * sp : s->species ) delete sp;
    delete s;
}

/* bc: {xlo, xhi, ylo, yhi} species::bc values or nullptr to keep defaults */
int ref_add_species( void * h, const char * name, float m_q, unsigned ppcx, unsigned ppcy,
                     int dens_type, const float * dens_p,
                     int udist_type, const float * uth, const float * ufl, int npmin,
                     int push_type, const int * bc ) {
    RefSim * s = static_cast<RefSim *>( h );
    HSpecies * sp = new HSpecies( name, m_q, make_uint2( ppcx, ppcy ) );
    Density::Profile * d = make_density( dens_type, dens_p );
    UDistribution::Type * u = make_udist( udist_type, uth, ufl, npmin );
    if ( !d || !u ) { delete sp; delete d; delete u; return -1; }
    sp->set_density( *d ); delete d;
    sp->set_udist( *u );   delete u;
    sp->push_type = push_type ? species::euler : species::boris;
    if ( bc ) {
        species::bc_type b;
        b.x.lower = (species::bc::type) bc[0]; b.x.upper = (species::bc::type) bc[1];
        b.y.lower = (species::bc::type) bc[2]; b.y.upper = (species::bc::type) bc[3];
        sp->set_bc( b );
    }
    s->species.push_back( sp );
    s->sim->add_species( *sp );
    return (int) s->species.size() - 1;
}

void ref_set_moving_window( void * h ) { static_cast<RefSim *>( h )->sim->set_moving_window(); }

void ref_emf_set_bc( void * h, const int * bc ) {
    emf::bc_type b;
    b.x.lower = (emf::bc::type) bc[0]; b.x.upper = (emf::bc::type) bc[1];
    b.y.lower = (emf::bc::type) bc[2]; b.y.upper = (emf::bc::type) bc[3];
    static_cast<RefSim *>( h )->sim->emf.set_bc( b );
}

void ref_current_set_bc( void * h, const int * bc ) {
    current::bc_type b;
    b.x.lower = (current::bc::type) bc[0]; b.x.upper = (current::bc::type) bc[1];
    b.y.lower = (current::bc::type) bc[2]; b.y.upper = (current::bc::type) bc[3];
    static_cast<RefSim *>( h )->sim->current.set_bc( b );
}

/* type: 0 none, 1 binomial, 2 compensated; dir 0 x / 1 y */
void ref_current_set_filter( void * h, int type, int dir, unsigned order ) {
    RefSim * s = static_cast<RefSim *>( h );
    coord::cart d = dir ? coord::y : coord::x;
    if ( type == 1 )      s->sim->current.set_filter( Filter::Binomial( d, order ) );
    else if ( type == 2 ) s->sim->current.set_filter( Filter::Compensated( d, order ) );
    else                  s->sim->current.set_filter( Filter::None() );
}

/*
 * p = { start, fwhm, rise, flat, fall, a0, omega0, polarization,
 *       cos_pol, sin_pol, filter, W0, focus, axis }
 * type 0 plane wave, 1 gaussian
 */
int ref_add_laser( void * h, int type, const float * p ) {
    RefSim * s = static_cast<RefSim *>( h );
    Laser::Pulse * l;
    if ( type == 0 ) l = new Laser::PlaneWave();
    else {
        Laser::Gaussian * g = new Laser::Gaussian();
        g->W0 = p[11]; g->focus = p[12]; g->axis = p[13];
        l = g;
    }
    l->start = p[0]; l->fwhm = p[1]; l->rise = p[2]; l->flat = p[3]; l->fall = p[4];
    l->a0 = p[5]; l->omega0 = p[6]; l->polarization = p[7];
    l->cos_pol = p[8]; l->sin_pol = p[9]; l->filter = (unsigned) p[10];
    int ierr = l->add( s->sim->emf );
    delete l;
    return ierr;
}

void ref_advance( void * h, int n ) {
    RefSim * s = static_cast<RefSim *>( h );
    for ( int i = 0; i < n; i++ ) s->sim->advance();
}

void ref_advance_mov_window( void * h, int n ) {
    RefSim * s = static_cast<RefSim *>( h );
    for ( int i = 0; i < n; i++ ) s->sim->advance_mov_window();
}

/* Fine-grained pieces of Simulation::advance (simulation.h:90-107) */
void ref_current_zero( void * h )    { static_cast<RefSim *>( h )->sim->current.zero(); }
void ref_current_advance( void * h ) { static_cast<RefSim *>( h )->sim->current.advance(); }
void ref_emf_advance( void * h, int with_current ) {
    RefSim * s = static_cast<RefSim *>( h );
    if ( with_current ) s->sim->emf.advance( s->sim->current );
    else s->sim->emf.advance();
}
void ref_species_advance( void * h, int sp ) {
    RefSim * s = static_cast<RefSim *>( h );
    s->species[sp]->advance( s->sim->emf, s->sim->current );
}
void ref_species_advance_free( void * h, int sp ) {
    static_cast<RefSim *>( h )->species[sp]->advance();
}
void ref_species_push( void * h, int sp ) {
    RefSim * s = static_cast<RefSim *>( h );
    s->species[sp]->push( s->sim->emf.E, s->sim->emf.B );
}
void ref_species_move( void * h, int sp ) {
    RefSim * s = static_cast<RefSim *>( h );
    s->species[sp]->move( s->sim->current.J );
}
void ref_species_process_bc( void * h, int sp ) {
    static_cast<RefSim *>( h )->species[sp]->bc();
}
void ref_species_tile_sort( void * h, int sp ) {
    RefSim * s = static_cast<RefSim *>( h );
    HSpecies * p = s->species[sp];
    p->parts()->tile_sort( *p->tmp_parts(), *p->sorter() );
}

unsigned ref_iter( void * h ) { return static_cast<RefSim *>( h )->sim->get_iter(); }
uint64_t ref_nmove( void * h ) { return static_cast<RefSim *>( h )->sim->get_nmove(); }

double ref_species_energy( void * h, int sp ) {
    return static_cast<RefSim *>( h )->species[sp]->get_energy();
}

void ref_emf_energy( void * h, double * out6 ) {
    double3 e, b;
    static_cast<RefSim *>( h )->sim->emf.get_energy( e, b );
    out6[0] = e.x; out6[1] = e.y; out6[2] = e.z;
    out6[3] = b.x; out6[4] = b.y; out6[5] = b.z;
}

/* Tile information: np[ntiles], offset[ntiles]; returns total particles */
uint64_t ref_species_tiles( void * h, int sp, int * np, int * offset ) {
    Particles * p = static_cast<RefSim *>( h )->species[sp]->parts();
    unsigned nt = p->ntiles.x * p->ntiles.y;
    if ( np )     std::memcpy( np, p->np, nt * sizeof( int ) );
    if ( offset ) std::memcpy( offset, p->offset, nt * sizeof( int ) );
    return p->np_total();
}

uint32_t ref_species_max_part( void * h, int sp ) {
    return static_cast<RefSim *>( h )->species[sp]->parts()->max_part;
}

/* Particles copied tile by tile into packed arrays (ix: 2 ints, x: 2 floats, u: 3 floats) */
void ref_species_get( void * h, int sp, int * ix, float * x, float * u ) {
    Particles * p = static_cast<RefSim *>( h )->species[sp]->parts();
    unsigned nt = p->ntiles.x * p->ntiles.y;
    size_t k = 0;
    for ( unsigned t = 0; t < nt; t++ ) {
        for ( int i = 0; i < p->np[t]; i++, k++ ) {
            size_t j = p->offset[t] + i;
            ix[2*k] = p->ix[j].x; ix[2*k+1] = p->ix[j].y;
            x[2*k]  = p->x[j].x;  x[2*k+1]  = p->x[j].y;
            u[3*k]  = p->u[j].x;  u[3*k+1]  = p->u[j].y; u[3*k+2] = p->u[j].z;
        }
    }
}

/* Replace the particle set: np per tile, packed arrays (tiles contiguous, tile order) */
int ref_species_set( void * h, int sp, const int * np, const int * ix, const float * x, const float * u ) {
    Particles * p = static_cast<RefSim *>( h )->species[sp]->parts();
    unsigned nt = p->ntiles.x * p->ntiles.y;
    size_t total = 0;
    for ( unsigned t = 0; t < nt; t++ ) total += np[t];
    if ( total > p->max_part ) return -1;
    size_t off = 0;
    for ( unsigned t = 0; t < nt; t++ ) { p->offset[t] = off; p->np[t] = np[t]; off += np[t]; }
    for ( size_t k = 0; k < total; k++ ) {
        p->ix[k] = make_int2( ix[2*k], ix[2*k+1] );
        p->x[k]  = make_float2( x[2*k], x[2*k+1] );
        p->u[k]  = make_float3( u[3*k], u[3*k+1], u[3*k+2] );
    }
    return 0;
}

/* Full tiled buffer, guard cells included: buffer_size()*3 floats */
uint64_t ref_grid_size( void * h, int which ) {
    return pick_grid( static_cast<RefSim *>( h ), which )->buffer_size();
}
void ref_grid_get( void * h, int which, float * out ) {
    vec3grid<float3> * g = pick_grid( static_cast<RefSim *>( h ), which );
    std::memcpy( out, g->d_buffer, g->buffer_size() * sizeof( float3 ) );
}
void ref_grid_set( void * h, int which, const float * in ) {
    vec3grid<float3> * g = pick_grid( static_cast<RefSim *>( h ), which );
    std::memcpy( (void *) g->d_buffer, in, g->buffer_size() * sizeof( float3 ) );
}

/* ZDF diagnostics written by the reference itself (files under the current directory) */
void ref_emf_save( void * h, int field, int fc ) {
    static_cast<RefSim *>( h )->sim->emf.save( field ? emf::b : emf::e, (fcomp::cart) fc );
}
void ref_current_save( void * h, int fc ) {
    static_cast<RefSim *>( h )->sim->current.save( (fcomp::cart) fc );
}
void ref_species_save_charge( void * h, int sp ) {
    static_cast<RefSim *>( h )->species[sp]->save_charge();
}

/* Species::dep_phasespace, 1D or 2D (quant1 < 0 selects 1D) */
int ref_species_phasespace( void * h, int sp, int q0, const float * range0, int size0,
                            int q1, const float * range1, int size1, float * out ) {
    RefSim * s = static_cast<RefSim *>( h );
    HSpecies * p = s->species[sp];
    if ( q1 < 0 ) {
        p->dep_phasespace( out, (phasespace::quant) q0, make_float2( range0[0], range0[1] ), (unsigned) size0 );
    } else {
        if ( q0 >= q1 ) return -1;
        p->dep_phasespace( out, (phasespace::quant) q0, make_float2( range0[0], range0[1] ), (unsigned) size0,
                           (phasespace::quant) q1, make_float2( range1[0], range1[1] ), (unsigned) size1 );
    }
    return 0;
}

/* Charge density as Species::save_charge builds it (species.cpp:2499-2511), gathered dense */
void ref_species_charge( void * h, int sp, float * out ) {
    RefSim * s = static_cast<RefSim *>( h );
    HSpecies * p = s->species[sp];
    bnd<unsigned int> gc; gc.x = {0,1}; gc.y = {0,1};
    grid<float> charge( p->parts()->ntiles, p->parts()->nx, gc );
    charge.zero();
    p->deposit_charge( charge );
    charge.add_from_gc();
    charge.gather( out );
}

}
