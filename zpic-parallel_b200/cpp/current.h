// current.h -- Current (current.h:17-148 of the reference) over libzpic_b200.so
#ifndef ZPIC_B200_CURRENT_H_
#define ZPIC_B200_CURRENT_H_

#include "zpic.h"
#include "vec3grid.h"
#include "filter.h"
#include "moving_window.h"

namespace current {
namespace bc { enum type { none = 0, periodic, reflecting }; }
typedef bnd<bc::type> bc_type;
}

class Current {
    zpic_sim * h_;
    float2 dx;
    double dt;
    current::bc_type bc;
    int iter;
    MovingWindow moving_window;
public:
    vec3grid<float3> * J;
    const float2 box;
    Filter::Digital * filter;

    Current( zpic_sim * h, uint2 const ntiles, uint2 const nx, float2 const box, double const dt ) :
        h_( h ), dx( make_float2( box.x / ( nx.x * ntiles.x ), box.y / ( nx.y * ntiles.y ) ) ), dt( dt ),
        bc( current::bc::periodic ), iter( 0 ), box( box ) {
        J = new vec3grid<float3>( h, ZPIC_GRID_J, ntiles, nx );
        J->name = "Current density";
        filter = new Filter::None();
    }
    ~Current() { delete J; delete filter; }

    auto get_iter() { return iter; }
    auto get_dt() { return dt; }
    current::bc_type get_bc() { return bc; }

    void set_bc( current::bc_type new_bc ) {
        const int32_t b[4] = { new_bc.x.lower, new_bc.x.upper, new_bc.y.lower, new_bc.y.upper };
        zpic::check( zpic_b200_current_set_bc( h_, b ) );
        bc = new_bc;
        std::string bc_name[] = { "none", "periodic", "reflecting" };
        std::cout << "(*info*) Current boundary conditions\n";
        std::cout << "(*info*) x : [ " << bc_name[bc.x.lower] << ", " << bc_name[bc.x.upper] << " ]\n";
        std::cout << "(*info*) y : [ " << bc_name[bc.y.lower] << ", " << bc_name[bc.y.upper] << " ]\n";
    }

    // called by Simulation::set_moving_window (library state already switched)
    int set_moving_window() {
        if ( iter != 0 ) { std::cerr << "(*error*) set_moving_window() called with iter != 0\n"; return -1; }
        moving_window.init( dx.x );
        bc.x.lower = bc.x.upper = current::bc::none;
        return 0;
    }

    void set_filter( Filter::Digital const & f ) {
        delete filter;
        filter = f.clone();
        zpic::check( zpic_b200_current_set_filter( h_, filter->type(), (int32_t) filter->direction(), filter->get_order() ) );
    }

    void advance() {
        zpic::check( zpic_b200_current_advance( h_ ) );
        iter++;
        if ( moving_window.needs_move( iter * dt ) ) moving_window.advance();
    }
    void zero() { zpic::check( zpic_b200_current_zero( h_ ) ); }

    // Current::save (current.cpp:262-313), including its axis ranges
    void save( fcomp::cart const jc ) {
        const char comp[] = { 'x', 'y', 'z' };
        zdf::grid_info info;
        info.name = std::string( "J" ) + comp[jc];
        info.label = std::string( "J_" ) + comp[jc];
        info.units = "e \\omega_n^2 / c";
        info.axis = { { "x", 0, 0.0 + moving_window.motion(), box.x, "x", "c/\\omega_n" },
                      { "y", 0, 0.0 + moving_window.motion(), box.y, "y", "c/\\omega_n" } };
        zdf::iteration it; it.n = iter; it.t = iter * dt; it.time_units = "1/\\omega_n";
        J->save( jc, info, it, "CURRENT" );
    }

    void step_bookkeeping() { iter++; if ( moving_window.needs_move( iter * dt ) ) moving_window.advance(); }
};

#endif
