// fk_spline.h -- not-a-knot cubic spline of the E(t) samples (host, O(nt)).
//
// The reference evaluates E between samples with a not-a-knot cubic spline
// through (i*dt, Et[i]) (spline_cubic_set with ibc 3 at
// src/cuda/fk_grad_Et_mono_PARAMETERS.cu:1681, evaluated by spline_cubic_val2
// at :1694 and :1879).  This is an independent implementation from the
// second-derivative form of the spline (de Boor, "A Practical Guide to
// Splines", ch. IV): the interior continuity rows are tridiagonal; the two
// not-a-knot rows give ypp_0 and ypp_{n-1} in terms of their two neighbours
// and are eliminated into rows 1 and n-2, leaving a diagonally dominant
// tridiagonal system solved by the Thomas algorithm.  The transposed map
// (samples -> values at fixed offsets) backs the discrete-exact gradient.
#pragma once

#include <vector>

namespace fkadj {

class NakSpline {
public:
    // n knots t_i = i*dt; n >= 4.
    NakSpline(int n, double dt);
    bool ok() const { return n_ >= 4; }
    // second derivatives at the knots for samples y[0..n)
    void second_derivs(const double* y, double* ypp) const;
    // value at t of the spline with samples y and second derivatives ypp
    double value(const double* y, const double* ypp, double t) const;
    // gy += Phi^T g where Phi maps samples to the spline values at
    // t = (l + frac)*dt, l = 0..n-2.
    void transpose_add(double frac, const double* g, double* gy) const;

private:
    int n_;
    double dt_;
    std::vector<double> sub_, dia_, sup_;
    double e0a_, e0b_, e1a_, e1b_;
    double knot(int i) const { return (double)i * dt_; }
    void thomas(double* x, bool transposed) const;
    int interval(double t) const;
};

}  // namespace fkadj
