// fk_spline.cpp -- see fk_spline.h.
#include "fk_spline.h"

#include <cmath>

namespace fkadj {

NakSpline::NakSpline(int n, double dt) : n_(n), dt_(dt) {
    if (n < 4) return;
    const int m = n - 2;
    sub_.assign(m, 0.0);
    dia_.assign(m, 0.0);
    sup_.assign(m, 0.0);
    for (int r = 1; r <= n - 2; ++r) {
        sub_[r - 1] = (knot(r) - knot(r - 1)) / 6.0;
        dia_[r - 1] = (knot(r + 1) - knot(r - 1)) / 3.0;
        sup_[r - 1] = (knot(r + 1) - knot(r)) / 6.0;
    }
    // not-a-knot rows: third derivative continuous at t_1 and t_{n-2}
    const double h0 = knot(1) - knot(0), h1 = knot(2) - knot(1);
    e0a_ = (knot(2) - knot(0)) / h1;
    e0b_ = -h0 / h1;
    const double H1 = knot(n - 2) - knot(n - 3), H2 = knot(n - 1) - knot(n - 2);
    e1a_ = (knot(n - 1) - knot(n - 3)) / H1;
    e1b_ = -H2 / H1;
    dia_[0] += sub_[0] * e0a_;
    sup_[0] += sub_[0] * e0b_;
    sub_[0] = 0.0;
    dia_[m - 1] += sup_[m - 1] * e1a_;
    sub_[m - 1] += sup_[m - 1] * e1b_;
    sup_[m - 1] = 0.0;
}

void NakSpline::thomas(double* x, bool tr) const {
    const int m = n_ - 2;
    std::vector<double> c(m);
    for (int r = 0; r < m; ++r) {
        const double lo = tr ? (r > 0 ? sup_[r - 1] : 0.0) : sub_[r];
        const double up = tr ? (r + 1 < m ? sub_[r + 1] : 0.0) : sup_[r];
        const double den = dia_[r] - (r > 0 ? lo * c[r - 1] : 0.0);
        c[r] = up / den;
        x[r] = (x[r] - (r > 0 ? lo * x[r - 1] : 0.0)) / den;
    }
    for (int r = m - 2; r >= 0; --r) x[r] -= c[r] * x[r + 1];
}

void NakSpline::second_derivs(const double* y, double* ypp) const {
    double* x = ypp + 1;
    for (int r = 1; r <= n_ - 2; ++r) {
        const double hm = knot(r) - knot(r - 1), hp = knot(r + 1) - knot(r);
        x[r - 1] = (y[r + 1] - y[r]) / hp - (y[r] - y[r - 1]) / hm;
    }
    thomas(x, false);
    ypp[0] = e0a_ * ypp[1] + e0b_ * ypp[2];
    ypp[n_ - 1] = e1a_ * ypp[n_ - 2] + e1b_ * ypp[n_ - 3];
}

int NakSpline::interval(double t) const {
    int l = (int)std::floor(t / dt_);
    if (l < 0) l = 0;
    if (l > n_ - 2) l = n_ - 2;
    while (l > 0 && t < knot(l)) --l;
    while (l < n_ - 2 && t > knot(l + 1)) ++l;
    return l;
}

double NakSpline::value(const double* y, const double* ypp, double t) const {
    const int l = interval(t), r = l + 1;
    const double s = t - knot(l), h = knot(r) - knot(l);
    return y[l] + s * ((y[r] - y[l]) / h - (ypp[r] / 6.0 + ypp[l] / 3.0) * h +
                       s * (0.5 * ypp[l] + s * ((ypp[r] - ypp[l]) / (6.0 * h))));
}

void NakSpline::transpose_add(double frac, const double* g, double* gy) const {
    const int m = n_ - 2;
    std::vector<double> gp(n_, 0.0), x(m);
    for (int l = 0; l < n_ - 1; ++l) {
        const double t = ((double)l + frac) * dt_;
        const double s = t - knot(l), h = knot(l + 1) - knot(l);
        gy[l] += (1.0 - s / h) * g[l];
        gy[l + 1] += (s / h) * g[l];
        gp[l] += (-s * h / 3.0 + 0.5 * s * s - s * s * s / (6.0 * h)) * g[l];
        gp[l + 1] += (-s * h / 6.0 + s * s * s / (6.0 * h)) * g[l];
    }
    for (int r = 0; r < m; ++r) x[r] = gp[r + 1];
    x[0] += e0a_ * gp[0];
    x[1] += e0b_ * gp[0];
    x[m - 1] += e1a_ * gp[n_ - 1];
    x[m - 2] += e1b_ * gp[n_ - 1];
    thomas(x.data(), true);
    for (int r = 1; r <= n_ - 2; ++r) {
        const double hm = knot(r) - knot(r - 1), hp = knot(r + 1) - knot(r);
        const double gb = x[r - 1];
        gy[r + 1] += gb / hp;
        gy[r] -= gb / hp + gb / hm;
        gy[r - 1] += gb / hm;
    }
}

}  // namespace fkadj
