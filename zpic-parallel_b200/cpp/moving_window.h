// moving_window.h -- MovingWindow (moving_window.h:1-57 of the reference)
#ifndef ZPIC_B200_MOVING_WINDOW_H_
#define ZPIC_B200_MOVING_WINDOW_H_

class MovingWindow {
    bool active_;
    unsigned int n_move_;
    double dx_;
public:
    MovingWindow() : active_( false ), n_move_( 0 ), dx_( 0 ) {}
    void init( float const dx ) { active_ = true; n_move_ = 0; dx_ = dx; }
    bool active() const { return active_; }
    unsigned int n_move() const { return n_move_; }
    int advance() { if ( active_ ) n_move_++; return n_move_; }
    double motion() const { return n_move_ * dx_; }
    bool needs_move( double const t ) const { return active_ && ( t > dx_ * ( n_move_ + 1 ) ); }
};

#endif
