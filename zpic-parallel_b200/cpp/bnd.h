// bnd.h -- per-edge boundary values (the reference's openmp/em2d/bnd.h layout:
// x.lower, x.upper, y.lower, y.upper).
#ifndef ZPIC_B200_BND_H_
#define ZPIC_B200_BND_H_

namespace edge { enum pos { lower = 0, upper }; }

template < typename T >
class bnd {
public:
    struct { T lower; T upper; } x;
    struct { T lower; T upper; } y;
    bnd() : x( { static_cast<T>( 0 ), static_cast<T>( 0 ) } ), y( { static_cast<T>( 0 ), static_cast<T>( 0 ) } ) {}
    bnd( T val ) : x( { val, val } ), y( { val, val } ) {}
    friend bool operator==( const bnd & a, const bnd & b ) {
        return a.x.lower == b.x.lower && a.x.upper == b.x.upper && a.y.lower == b.y.lower && a.y.upper == b.y.upper;
    }
    friend bool operator!=( const bnd & a, const bnd & b ) { return !( a == b ); }
};

#endif
