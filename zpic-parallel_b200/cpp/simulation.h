// simulation.h -- Simulation (simulation.h:14-184 of the reference): one em2d
// simulation whose step runs on a B200 through libzpic_b200.so.  The public
// interface is the reference's; EMF, Current and Species are views of the
// library's device state.
#ifndef ZPIC_B200_SIMULATION_H_
#define ZPIC_B200_SIMULATION_H_

#include <vector>

#include "zpic.h"
#include "emf.h"
#include "current.h"
#include "species.h"
#include "laser.h"
#include "filter.h"

namespace detail {
inline zpic_sim * create_sim( uint2 ntiles, uint2 nx, float2 box, double dt ) {
    zpic_sim * h = nullptr;
    zpic::check( zpic_b200_sim_create( ntiles.x, ntiles.y, nx.x, nx.y, box.x, box.y, dt, &h ) );
    return h;
}
}

class Simulation {
    unsigned int iter;
    zpic_sim * h_;
public:
    const uint2 ntiles;
    const uint2 nx;
    const float2 box;
    const double dt;
    EMF emf;
    Current current;
    std::vector<Species *> species;

    Simulation( uint2 const ntiles, uint2 const nx, float2 const box, double dt ) :
        iter( 0 ), h_( detail::create_sim( ntiles, nx, box, dt ) ), ntiles( ntiles ), nx( nx ), box( box ), dt( dt ),
        emf( h_, ntiles, nx, box, dt ), current( h_, ntiles, nx, box, dt ) {}
    ~Simulation() { zpic_b200_sim_destroy( h_ ); }
    Simulation( const Simulation & ) = delete;
    Simulation & operator=( const Simulation & ) = delete;

    zpic_sim * handle() const { return h_; }

    void set_moving_window() {
        zpic::check( zpic_b200_sim_set_moving_window( h_ ) );
        emf.set_moving_window();
        current.set_moving_window();
        for ( auto * s : species ) s->set_moving_window();
    }

    void add_species( Species & s ) {
        species.push_back( &s );
        s.initialize( h_, box, ntiles, nx, dt, (int) species.size() );
    }

    Species * get_species( std::string name ) {
        for ( auto * s : species ) if ( s->name == name ) return s;
        return nullptr;
    }

    // Simulation::advance (simulation.h:90-107)
    void advance() {
        for ( auto * s : species ) s->sync_push_type();
        zpic::check( zpic_b200_sim_advance( h_, 1 ) );
        bookkeeping( false );
    }
    // several steps in one call (CUDA-graph replay)
    void advance( int nsteps ) {
        for ( auto * s : species ) s->sync_push_type();
        zpic::check( zpic_b200_sim_advance( h_, nsteps ) );
        for ( int n = 0; n < nsteps; n++ ) bookkeeping( false );
    }
    // Simulation::advance_mov_window (simulation.h:113-130)
    void advance_mov_window() {
        for ( auto * s : species ) s->sync_push_type();
        zpic::check( zpic_b200_sim_advance_mov_window( h_, 1 ) );
        bookkeeping( true );
    }

    unsigned int get_iter() { return iter; }
    double get_t() { return iter * double( dt ); }

    // Simulation::energy_info (simulation.h:150-170)
    void energy_info() {
        std::cout << "(*info*) Energy at n = " << iter << ", t = " << iter * double( dt ) << '\n';
        double part_ene = 0;
        for ( auto * s : species ) {
            double kin = s->get_energy();
            std::cout << "(*info*) " << s->name << " = " << kin << '\n';
            part_ene += kin;
        }
        if ( species.size() > 1 ) std::cout << "(*info*) Total particle energy = " << part_ene << '\n';
        double3 ene_E, ene_B;
        emf.get_energy( ene_E, ene_B );
        std::cout << "(*info*) Electric field = " << ene_E.x + ene_E.y + ene_E.z << '\n';
        std::cout << "(*info*) Magnetic field = " << ene_B.x + ene_B.y + ene_B.z << '\n';
        double total = part_ene + ene_E.x + ene_E.y + ene_E.z + ene_B.x + ene_B.y + ene_B.z;
        std::cout << "(*info*) total = " << total << '\n';
    }

    uint64_t get_nmove() {
        uint64_t n = 0;
        zpic::check( zpic_b200_sim_nmove( h_, &n ) );
        return n;
    }

private:
    void bookkeeping( bool mw ) {
        for ( auto * s : species ) s->step_bookkeeping( mw );
        current.step_bookkeeping();
        emf.step_bookkeeping();
        iter++;
    }
};

#endif
