// vec3grid.h -- host view of a tiled float3 grid that lives on the GPU
// (the reference's grid.h / vec3grid.h geometry: guard cells {1,2},
// tile_vol = roundup4(ext_x * ext_y)).
#ifndef ZPIC_B200_VEC3GRID_H_
#define ZPIC_B200_VEC3GRID_H_

#include <vector>

#include "zpic.h"
#include "zdf.h"

template < class V >
class vec3grid {
    zpic_sim * h_;
    int which_;
public:
    const uint2 ntiles, nx, dims, ext_nx;
    const bnd<unsigned int> gc;
    const unsigned int offset, tile_vol;
    std::string name;

    vec3grid( zpic_sim * h, int which, uint2 ntiles_, uint2 nx_ ) :
        h_( h ), which_( which ), ntiles( ntiles_ ), nx( nx_ ),
        dims( make_uint2( ntiles_.x * nx_.x, ntiles_.y * nx_.y ) ),
        ext_nx( make_uint2( 1 + nx_.x + 2, 1 + nx_.y + 2 ) ), gc( 0 ),
        offset( 1 * ( 1 + nx_.x + 2 ) + 1 ),
        tile_vol( ( ( 1 + nx_.x + 2 ) * ( 1 + nx_.y + 2 ) + 3 ) & ~3u ) {
        const_cast<bnd<unsigned int> &>( gc ).x = { 1, 2 };
        const_cast<bnd<unsigned int> &>( gc ).y = { 1, 2 };
    }

    std::size_t buffer_size() const { return (std::size_t) tile_vol * ntiles.x * ntiles.y; }

    // vec3grid::gather (vec3grid.h:76-205): one component, dense grid
    unsigned int gather( const enum fcomp::cart fc, float * const out ) const {
        zpic::check( zpic_b200_grid_gather( h_, which_, (int32_t) fc, out ) );
        return dims.x * dims.y;
    }

    // the whole tiled buffer (guard cells included), copied from / to the GPU
    std::vector<V> get() const {
        std::vector<V> v( buffer_size() );
        zpic::check( zpic_b200_grid_get( h_, which_, reinterpret_cast<float *>( v.data() ) ) );
        return v;
    }
    void set( const std::vector<V> & v ) {
        zpic::check( zpic_b200_grid_set( h_, which_, reinterpret_cast<const float *>( v.data() ) ) );
    }

    // vec3grid::save (vec3grid.h:398-420)
    void save( const enum fcomp::cart fc, zdf::grid_info & info, zdf::iteration & iter, const std::string & path ) const {
        info.ndims = 2; info.count[0] = dims.x; info.count[1] = dims.y;
        std::vector<float> buf( (size_t) dims.x * dims.y );
        gather( fc, buf.data() );
        zdf::save_grid( buf.data(), info, iter, path );
    }
};

#endif
