// filter.h -- Filter::{None, Binomial, Compensated} (filter.h:9-86 of the reference)
#ifndef ZPIC_B200_FILTER_H_
#define ZPIC_B200_FILTER_H_

#include "zpic.h"

namespace Filter {

class Digital {
public:
    virtual Digital * clone() const = 0;
    virtual int type() const = 0;
    virtual coord::cart direction() const { return coord::x; }
    virtual unsigned int get_order() const { return 1; }
    virtual ~Digital() = default;
};

class None : public Digital {
public:
    None * clone() const override { return new None(); }
    int type() const override { return ZPIC_FILTER_NONE; }
};

class Binomial : public Digital {
protected:
    unsigned int order; coord::cart dir;
public:
    Binomial( coord::cart dir, unsigned int order = 0 ) : order( ( order > 0 ) ? order : 1 ), dir( dir ) {}
    Binomial * clone() const override { return new Binomial( dir, order ); }
    int type() const override { return ZPIC_FILTER_BINOMIAL; }
    coord::cart direction() const override { return dir; }
    unsigned int get_order() const override { return order; }
};

class Compensated : public Binomial {
public:
    Compensated( coord::cart dir, unsigned int order = 0 ) : Binomial( dir, order ) {}
    Compensated * clone() const override { return new Compensated( dir, order ); }
    int type() const override { return ZPIC_FILTER_COMPENSATED; }
};

}  // namespace Filter

#endif
