// species.h -- Species (species.h:55-528 of the reference) over libzpic_b200.so
#ifndef ZPIC_B200_SPECIES_H_
#define ZPIC_B200_SPECIES_H_

#include <string>
#include <vector>

#include "zpic.h"
#include "emf.h"
#include "current.h"
#include "density.h"
#include "udist.h"
#include "moving_window.h"

namespace species {
enum pusher { boris, euler };
namespace bc { enum type { open = 0, periodic, reflecting }; }
typedef bnd<bc::type> bc_type;
}

namespace phasespace {
enum quant { x, y, ux, uy, uz };
static inline void qinfo( quant q, std::string & name, std::string & label, std::string & units ) {
    switch ( q ) {
    case x: name = "x"; label = "x"; units = "c/\\omega_n"; break;
    case y: name = "y"; label = "y"; units = "c/\\omega_n"; break;
    case ux: name = "ux"; label = "u_x"; units = "c"; break;
    case uy: name = "uy"; label = "u_y"; units = "c"; break;
    case uz: name = "uz"; label = "u_z"; units = "c"; break;
    }
}
}

class Species {
    zpic_sim * h_ = nullptr;
    int index_ = -1;
    int id = 0;
    uint2 ppc;
    float q = 0;
    float2 dx = { 0, 0 }, box = { 0, 0 };
    float dt = 0;
    int iter = 0;
    Density::Profile * density;
    UDistribution::Type * udist;
    species::bc_type bc;
    MovingWindow moving_window;
    uint2 ntiles_ = { 0, 0 }, nx_ = { 0, 0 };

    zpic_species_desc desc() const {
        zpic_species_desc d{};
        d.name = name.c_str();
        d.m_q = m_q;
        d.ppc[0] = ppc.x; d.ppc[1] = ppc.y;
        d.density = density->desc();
        d.udist = udist->desc();
        d.push_type = push_type;
        d.bc[0] = bc.x.lower; d.bc[1] = bc.x.upper; d.bc[2] = bc.y.lower; d.bc[3] = bc.y.upper;
        return d;
    }
    void attached() const {
        if ( !h_ ) { std::cerr << "(*error*) species " << name << " has not been added to a simulation\n"; std::exit( 1 ); }
    }

public:
    const std::string name;
    const float m_q;
    species::pusher push_type;

    // Species( name, m_q, ppc ) (species.cpp:1693-1718)
    Species( std::string const name, float const m_q, uint2 const ppc ) : ppc( ppc ), name( name ), m_q( m_q ) {
        if ( m_q == 0 ) { std::cerr << "(*error*) Invalid m_q value, must be not 0, aborting...\n"; std::exit( 1 ); }
        if ( ppc.x < 1 || ppc.y < 1 ) { std::cerr << "(*error*) Invalid ppc value, must be >= 1 in all directions\n"; std::exit( 1 ); }
        density = new Density::Uniform( 1.0 );
        udist = new UDistribution::None();
        bc = species::bc_type( species::bc::periodic );
        push_type = species::boris;
    }
    virtual ~Species() { delete density; delete udist; }

    // Species::initialize (species.cpp:1730-1788): called by Simulation::add_species
    virtual void initialize( zpic_sim * h, float2 const box_, uint2 const ntiles, uint2 const nx, double const dt_, int const id_ ) {
        zpic_species_desc d = desc();
        int32_t idx = -1;
        zpic::check( zpic_b200_sim_add_species( h, &d, &idx ) );
        h_ = h; index_ = idx; id = id_;
        box = box_; dt = dt_; ntiles_ = ntiles; nx_ = nx;
        q = std::copysign( density->n0, m_q ) / ( ppc.x * ppc.y );
        dx = make_float2( box.x / ( nx.x * ntiles.x ), box.y / ( nx.y * ntiles.y ) );
        iter = 0;
    }

    virtual void set_density( Density::Profile const & d ) { delete density; density = d.clone(); }
    Density::Profile & get_density() { return *density; }
    virtual void set_udist( UDistribution::Type const & u ) { delete udist; udist = u.clone(); }
    UDistribution::Type & get_udist() { return *udist; }

    void set_bc( species::bc_type new_bc ) {
        for ( int a = 0; a < 2; a++ ) {
            const auto lo = a ? new_bc.y.lower : new_bc.x.lower, hi = a ? new_bc.y.upper : new_bc.x.upper;
            if ( ( lo == species::bc::periodic || hi == species::bc::periodic ) && lo != hi ) {
                std::cerr << "(*error*) Species boundary type mismatch along " << ( a ? 'y' : 'x' ) << ".\n";
                std::exit( 1 );
            }
        }
        bc = new_bc;
        if ( h_ ) {
            const int32_t b[4] = { bc.x.lower, bc.x.upper, bc.y.lower, bc.y.upper };
            zpic::check( zpic_b200_species_set_bc( h_, index_, b ) );
        }
    }
    species::bc_type get_bc() { return bc; }

    virtual int set_moving_window() {
        if ( iter != 0 ) { std::cerr << "(*error*) set_moving_window() called with iter != 0\n"; return -1; }
        moving_window.init( dx.x );
        bc.x.lower = bc.x.upper = species::bc::open;
        return 0;
    }

    void sync_push_type() {
        if ( h_ ) zpic::check( zpic_b200_species_set_push_type( h_, index_, push_type ) );
    }

    void push( vec3grid<float3> * const, vec3grid<float3> * const ) { attached(); sync_push_type(); zpic::check( zpic_b200_species_push( h_, index_ ) ); }
    void move( vec3grid<float3> * const ) { attached(); zpic::check( zpic_b200_species_move( h_, index_ ) ); }

    virtual void advance() { attached(); zpic::check( zpic_b200_species_advance( h_, index_, ZPIC_ADVANCE_FREE ) ); iter++; }
    virtual void advance( Current & ) { attached(); zpic::check( zpic_b200_species_advance( h_, index_, ZPIC_ADVANCE_CURRENT ) ); iter++; }
    virtual void advance( EMF const &, Current & ) {
        attached(); sync_push_type();
        zpic::check( zpic_b200_species_advance( h_, index_, ZPIC_ADVANCE_FULL ) );
        iter++;
    }
    virtual void advance_mov_window( EMF const &, Current & ) {
        attached(); sync_push_type();
        const bool moved = moving_window.needs_move( ( iter + 1 ) * dt );
        zpic::check( zpic_b200_species_advance_mov_window( h_, index_ ) );
        if ( moved ) moving_window.advance();
        iter++;
    }
    // bookkeeping when the Simulation advanced the species
    void step_bookkeeping( bool mov_window ) {
        if ( mov_window && moving_window.needs_move( ( iter + 1 ) * dt ) ) moving_window.advance();
        iter++;
    }

    double get_energy() const {
        attached();
        double e = 0;
        zpic::check( zpic_b200_species_energy( h_, index_, &e ) );
        return e;
    }
    uint64_t get_nmove() const {
        attached();
        uint64_t n = 0;
        zpic::check( zpic_b200_species_nmove( h_, index_, &n ) );
        return n;
    }
    auto get_iter() const { return iter; }
    auto get_dt() const { return dt; }
    auto get_ntiles() const { return ntiles_; }
    auto get_nx() const { return nx_; }
    auto get_box() const { return box; }
    uint32_t np_max_tile() const { attached(); uint32_t n = 0; zpic::check( zpic_b200_species_np_max_tile( h_, index_, &n ) ); return n; }
    uint64_t np_total() const { attached(); uint64_t n = 0; zpic::check( zpic_b200_species_np_total( h_, index_, &n ) ); return n; }

    // Species::gather (species.h:510-526): positions in simulation units
    void gather( part::quant quant, float * const d_data ) {
        attached();
        zpic::check( zpic_b200_species_gather( h_, index_, (int32_t) quant, d_data ) );
    }

    // Species::save (species.cpp:2416-2480): x, y, ux, uy, uz in simulation units
    void save() {
        const uint64_t np = np_total();
        zdf::part_info info;
        info.name = name; info.label = name; info.np = np;
        info.quants = { "x", "y", "ux", "uy", "uz" };
        info.qlabels = { "x", "y", "u_x", "u_y", "u_z" };
        info.qunits = { "c/\\omega_n", "c/\\omega_n", "c", "c", "c" };
        zdf::iteration it; it.n = iter; it.t = iter * dt; it.time_units = "1/\\omega_n";
        std::vector<std::vector<float>> data( 5, std::vector<float>( np ) );
        for ( int k = 0; k < 5; k++ ) if ( np ) gather( (part::quant) k, data[k].data() );
        zdf::save_particles( info, it, "PARTICLES", data );
    }

    // Species::save_charge (species.cpp:2486-2549)
    void save_charge() {
        attached();
        std::vector<float> rho( (size_t) ntiles_.x * nx_.x * ntiles_.y * nx_.y );
        zpic::check( zpic_b200_species_charge( h_, index_, rho.data() ) );
        zdf::grid_info info;
        info.name = name + "-charge";
        info.label = name + " \\rho";
        info.units = "n_e";
        info.ndims = 2; info.count[0] = ntiles_.x * nx_.x; info.count[1] = ntiles_.y * nx_.y;
        info.axis = { { "x", 0, 0. + moving_window.motion(), box.x + moving_window.motion(), "x", "c/\\omega_n" },
                      { "y", 0, 0., box.y, "y", "c/\\omega_n" } };
        zdf::iteration it; it.name = "ITERATION"; it.n = iter; it.t = iter * dt; it.time_units = "1/\\omega_n";
        zdf::save_grid( rho.data(), info, it, "CHARGE/" + name );
    }

    // Species::dep_phasespace 1D / 2D (species.cpp:2631-2709, 2863-3022):
    // phase-space density into a host buffer of size0 (x size1) floats
    void dep_phasespace( float * const d_data, phasespace::quant q, float2 const range, unsigned const size ) const {
        attached();
        const float r[2] = { range.x, range.y };
        zpic::check( zpic_b200_species_phasespace( h_, index_, (int32_t) q, r, (int32_t) size, -1, nullptr, 0, d_data ) );
    }
    void dep_phasespace( float * const d_data, phasespace::quant quant0, float2 range0, unsigned const size0,
                         phasespace::quant quant1, float2 range1, unsigned const size1 ) const {
        attached();
        const float r0[2] = { range0.x, range0.y }, r1[2] = { range1.x, range1.y };
        zpic::check( zpic_b200_species_phasespace( h_, index_, (int32_t) quant0, r0, (int32_t) size0,
                                                   (int32_t) quant1, r1, (int32_t) size1, d_data ) );
    }

    // Species::save_phasespace 1D (species.cpp:2717-2765): PHASESPACE/<name>/<name>-<q>-<iter>.zdf
    void save_phasespace( phasespace::quant quant, float2 const range, int const size ) const {
        std::string qname, qlabel, qunits;
        phasespace::qinfo( quant, qname, qlabel, qunits );
        zdf::grid_info info;
        info.name = name + "-" + qname;
        info.label = name + "\\,(" + qlabel + ")";
        info.units = "n_e";
        info.ndims = 1; info.count[0] = size;
        const double shift = quant == phasespace::x ? moving_window.motion() : 0.0;
        info.axis = { { qname, 0, range.x + shift, range.y + shift, qlabel, qunits } };
        std::vector<float> data( size );
        dep_phasespace( data.data(), quant, range, size );
        zdf::iteration it; it.name = "ITERATION"; it.n = iter; it.t = iter * dt; it.time_units = "1/\\omega_n";
        zdf::save_grid( data.data(), info, it, "PHASESPACE/" + name );
    }

    // Species::save_phasespace 2D (species.cpp:3035-3105); quant1 must be indexed above quant0
    void save_phasespace( phasespace::quant quant0, float2 const range0, int const size0,
                          phasespace::quant quant1, float2 const range1, int const size1 ) const {
        if ( quant0 >= quant1 ) {
            std::cerr << "(*error*) for 2D phasespaces, the 2nd quantity must be indexed higher than the first one\n";
            return;
        }
        std::string qn0, ql0, qu0, qn1, ql1, qu1;
        phasespace::qinfo( quant0, qn0, ql0, qu0 );
        phasespace::qinfo( quant1, qn1, ql1, qu1 );
        zdf::grid_info info;
        info.name = name + "-" + qn0 + qn1;
        info.label = name + " \\,(" + ql0 + "\\rm{-}" + ql1 + ")";
        info.units = "n_e";
        info.ndims = 2; info.count[0] = size0; info.count[1] = size1;
        const double shift = quant0 == phasespace::x ? moving_window.motion() : 0.0;
        info.axis = { { qn0, 0, range0.x + shift, range0.y + shift, ql0, qu0 },
                      { qn1, 0, range1.x, range1.y, ql1, qu1 } };
        std::vector<float> data( (size_t) size0 * size1 );
        dep_phasespace( data.data(), quant0, range0, size0, quant1, range1, size1 );
        zdf::iteration it; it.name = "ITERATION"; it.n = iter; it.t = iter * dt; it.time_units = "1/\\omega_n";
        zdf::save_grid( data.data(), info, it, "PHASESPACE/" + name );
    }

    int index() const { return index_; }
};

#endif
