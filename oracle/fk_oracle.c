/*
 * fk_oracle.c -- CPU oracle (C99 + OpenMP, FP64) for the Fenton-Karma
 * forward RK4 sweep and the two adjoint gradients.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library, never shipped
 * or called by the product path.  Built with -ffp-contract=off so that every
 * expression rounds exactly as written; the expressions below keep the
 * reference's operation order (so that the only systematic difference to
 * the reference GPU build is FMA contraction and the libm tanh).
 *
 * Reference (agarzon27/adjoint-optimization), cited by file:line:
 *   cu-F = src/cuda/fk_forward_Et_mono_PARAMETERS.cu
 *   cu-G = src/cuda/fk_grad_Et_mono_PARAMETERS.cu
 */
#include "fk_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

void ora_set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

int ora_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------ model */

/* Ionic currents of the FK model; formula of cu-F:29-45. */
static void fk_ion(const ora_params *P, double u, double v, double w,
                   double *ud, double *vd, double *wd) {
    double p = 0.5 * (1 + tanh(P->ksm * (u - P->u_c)));
    double q = 0.5 * (1 + tanh(P->ksm * (u - P->u_v)));
    double j_fi = -v * p * (1 - u) * (u - P->u_c) / P->tau_d;
    double j_so = u * (1 - p) / P->tau_0 + p / P->tau_r;
    double tvm = q * P->tau_v1_minus + (1 - q) * P->tau_v2_minus;
    double j_si = -w * (1 + tanh(P->k_fk * (u - P->u_csi))) / (2 * P->tau_si);
    *ud = -(j_fi + j_so + j_si);
    *vd = ((1 - p) * (1 - v) / tvm) - (p * v) / P->tau_v_plus;
    *wd = ((1 - p) * (1 - w) / P->tau_w_minus) - (p * w) / P->tau_w_plus;
}

/* Transposed 3x3 Jacobian of fk_ion at (u,v,w), stored so that
 * (J^T z)_r = sum_c jt[3r+c] z_c; formula of cu-G:1160-1184. */
static void fk_ion_jacT(const ora_params *P, double u, double v, double w, double jt[9]) {
    double tc = tanh(P->ksm * (u - P->u_c));
    double tv = tanh(P->ksm * (u - P->u_v));
    double ts = tanh(P->k_fk * (u - P->u_csi));
    double p = 0.5 * tc + 0.5;
    double q = 0.5 * tv + 0.5;
    double dp = 1 - tc * tc;
    double dq = 1 - tv * tv;
    double tvm = q * P->tau_v1_minus + P->tau_v2_minus * (1 - q);
    double ksm = P->ksm;
    jt[0] = -0.5 * dp * ksm / P->tau_r + 0.5 * dp * ksm * v * (1 - u) * (u - P->u_c) / P->tau_d
          + 0.5 * dp * ksm * u / P->tau_0 + P->k_fk * w * (1 - ts * ts) / (2 * P->tau_si)
          + p * v * (1 - u) / P->tau_d - p * v * (u - P->u_c) / P->tau_d - (1 - p) / P->tau_0;
    jt[3] = p * (1 - u) * (u - P->u_c) / P->tau_d;
    jt[6] = (ts + 1) / (2 * P->tau_si);
    jt[1] = -0.5 * dp * ksm * v / P->tau_v_plus - 0.5 * dp * ksm * (1 - v) / tvm
          + (1 - p) * (1 - v) * (-0.5 * dq * ksm * P->tau_v1_minus + 0.5 * dq * ksm * P->tau_v2_minus)
            / (tvm * tvm);
    jt[4] = -p / P->tau_v_plus - (1 - p) / tvm;
    jt[7] = 0.0;
    jt[2] = -0.5 * dp * ksm * w / P->tau_w_plus - 0.5 * dp * ksm * (1 - w) / P->tau_w_minus;
    jt[5] = 0.0;
    jt[8] = -p / P->tau_w_plus - (1 - p) / P->tau_w_minus;
}

/* Neighbour indices the 5-point stencil uses at (i,j): grid edges mirror the
 * inner neighbour, a hole (NaN in u) is replaced by the opposite neighbour
 * (cu-F:319-420). */
static void stencil_nbrs(const double *u, int nrows, int ncols, int i, int j,
                         int *kim, int *kip, int *kjm, int *kjp) {
    int k = i * ncols + j;
    if (i == 0) {
        *kim = *kip = k + ncols;
    } else if (i == nrows - 1) {
        *kim = *kip = k - ncols;
    } else {
        *kim = k - ncols;
        *kip = k + ncols;
        if (isnan(u[*kim])) *kim = *kip;
        else if (isnan(u[*kip])) *kip = *kim;
    }
    if (j == 0) {
        *kjm = *kjp = k + 1;
    } else if (j == ncols - 1) {
        *kjm = *kjp = k - 1;
    } else {
        *kjm = k - 1;
        *kjp = k + 1;
        if (isnan(u[*kjm])) *kjm = *kjp;
        else if (isnan(u[*kjp])) *kjp = *kjm;
    }
}

void ora_rhs(const ora_params *P, int nrows, int ncols, const double *y,
             const double *gh, double E, double *f) {
    const int n = nrows * ncols;
    const double *u = y, *v = y + n, *w = y + 2 * n;
    double *fu = f, *fv = f + n, *fw = f + 2 * n;
    const double cu = P->Du / (P->h * P->h);
    const double cv = P->Dv / (P->h * P->h);
    const double cw = P->Dw / (P->h * P->h);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nrows; i++) {
        for (int j = 0; j < ncols; j++) {
            int k = i * ncols + j;
            if (isnan(u[k])) {
                fu[k] = fv[k] = fw[k] = NAN;
                continue;
            }
            int a, b, c, d;
            stencil_nbrs(u, nrows, ncols, i, j, &a, &b, &c, &d);
            double lu = cu * (u[a] + u[b] + u[c] + u[d] - 4.0 * u[k]);
            double lv = cv * (v[a] + v[b] + v[c] + v[d] - 4.0 * v[k]);
            double lw = cw * (w[a] + w[b] + w[c] + w[d] - 4.0 * w[k]);
            double ud, vd, wd;
            fk_ion(P, u[k], v[k], w[k], &ud, &vd, &wd);
            fu[k] = lu + ud + E * gh[k];
            fv[k] = lv + vd;
            fw[k] = lw + wd;
        }
    }
}

/* Weight with which a neighbour enters L^T: 0 when the neighbour is missing
 * (off-grid or hole), 2 when the neighbour's own far neighbour is missing
 * (it mirrored this cell), else 1 (cu-G:1004-1111). */
static double lapT_weight(const double *zu, int nrows, int ncols, int i, int j,
                          int di, int dj) {
    int i1 = i + di, j1 = j + dj, i2 = i + 2 * di, j2 = j + 2 * dj;
    if (i1 < 0 || i1 >= nrows || j1 < 0 || j1 >= ncols) return 0.0;
    if (isnan(zu[i1 * ncols + j1])) return 0.0;
    if (i2 < 0 || i2 >= nrows || j2 < 0 || j2 >= ncols) return 2.0;
    if (isnan(zu[i2 * ncols + j2])) return 2.0;
    return 1.0;
}

void ora_adj_rhs(const ora_params *P, int nrows, int ncols, const double *z,
                 const double *y, double *fz) {
    const int n = nrows * ncols;
    const double coef[3] = {P->Du / (P->h * P->h), P->Dv / (P->h * P->h), P->Dw / (P->h * P->h)};
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nrows; i++) {
        for (int j = 0; j < ncols; j++) {
            int k = i * ncols + j;
            if (isnan(z[k])) {
                fz[k] = fz[n + k] = fz[2 * n + k] = NAN;
                continue;
            }
            double pt = lapT_weight(z, nrows, ncols, i, j, -1, 0);
            double pb = lapT_weight(z, nrows, ncols, i, j, +1, 0);
            double pl = lapT_weight(z, nrows, ncols, i, j, 0, -1);
            double pr = lapT_weight(z, nrows, ncols, i, j, 0, +1);
            double lt[3];
            for (int c = 0; c < 3; c++) {
                const double *zc = z + (size_t)c * n;
                double vt = pt != 0.0 ? zc[k - ncols] : 0.0;
                double vb = pb != 0.0 ? zc[k + ncols] : 0.0;
                double vl = pl != 0.0 ? zc[k - 1] : 0.0;
                double vr = pr != 0.0 ? zc[k + 1] : 0.0;
                lt[c] = coef[c] * (pt * vt + pb * vb + pl * vl + pr * vr - 4.0 * zc[k]);
            }
            double jt[9];
            fk_ion_jacT(P, y[k], y[n + k], y[2 * n + k], jt);
            double zk[3] = {z[k], z[n + k], z[2 * n + k]};
            for (int r = 0; r < 3; r++) {
                double s = 0.0;
                for (int c = 0; c < 3; c++) s += jt[3 * r + c] * zk[c];
                fz[(size_t)r * n + k] = lt[r] + s;
            }
        }
    }
}

/* ----------------------------------------------------------------- spline */
/*
 * Not-a-knot cubic spline in second-derivative form (de Boor, "A Practical
 * Guide to Splines", ch. IV).  Knots t_i = i*dt.  The interior continuity
 * rows are tridiagonal; the two not-a-knot rows express ypp_0 and ypp_{n-1}
 * through their two neighbours, which are substituted into rows 1 and n-2 so
 * that a diagonally dominant tridiagonal system in ypp_1..ypp_{n-2} remains.
 * (The reference solves the same equations as a pentadiagonal system,
 * cu-F:1134-1427.)
 */
typedef struct {
    int n;                 /* knots */
    double *sub, *dia, *sup; /* reduced tridiagonal rows 1..n-2 (length n-2) */
    double e0a, e0b;       /* ypp_0     = e0a*ypp_1     + e0b*ypp_2     */
    double e1a, e1b;       /* ypp_{n-1} = e1a*ypp_{n-2} + e1b*ypp_{n-3} */
} nak_sys;

static double knot(int i, double dt) { return (double)i * dt; }

static int nak_build(int n, double dt, nak_sys *S) {
    if (n < 4) return -1;
    int m = n - 2;
    S->n = n;
    S->sub = (double *)calloc((size_t)m, sizeof(double));
    S->dia = (double *)calloc((size_t)m, sizeof(double));
    S->sup = (double *)calloc((size_t)m, sizeof(double));
    for (int r = 1; r <= n - 2; r++) {
        double hm = knot(r, dt) - knot(r - 1, dt), hp = knot(r + 1, dt) - knot(r, dt);
        S->sub[r - 1] = hm / 6.0;
        S->dia[r - 1] = (knot(r + 1, dt) - knot(r - 1, dt)) / 3.0;
        S->sup[r - 1] = hp / 6.0;
    }
    double h0 = knot(1, dt) - knot(0, dt), h1 = knot(2, dt) - knot(1, dt);
    S->e0a = (knot(2, dt) - knot(0, dt)) / h1;
    S->e0b = -h0 / h1;
    double H1 = knot(n - 2, dt) - knot(n - 3, dt), H2 = knot(n - 1, dt) - knot(n - 2, dt);
    S->e1a = (knot(n - 1, dt) - knot(n - 3, dt)) / H1;
    S->e1b = -H2 / H1;
    /* substitute ypp_0 into row 1 and ypp_{n-1} into row n-2 */
    S->dia[0] += S->sub[0] * S->e0a;
    S->sup[0] += S->sub[0] * S->e0b;
    S->sub[0] = 0.0;
    S->dia[m - 1] += S->sup[m - 1] * S->e1a;
    S->sub[m - 1] += S->sup[m - 1] * S->e1b;
    S->sup[m - 1] = 0.0;
    return 0;
}

static void nak_free(nak_sys *S) {
    free(S->sub);
    free(S->dia);
    free(S->sup);
}

/* Thomas solve of the reduced system (transposed when tr != 0), in place. */
static void nak_thomas(const nak_sys *S, double *x, int tr) {
    int m = S->n - 2;
    double *c = (double *)malloc((size_t)m * sizeof(double));
    /* row r: lo[r]*x[r-1] + dia[r]*x[r] + up[r]*x[r+1] */
    for (int r = 0; r < m; r++) {
        double lo = tr ? (r > 0 ? S->sup[r - 1] : 0.0) : S->sub[r];
        double up = tr ? (r + 1 < m ? S->sub[r + 1] : 0.0) : S->sup[r];
        double den = S->dia[r] - (r > 0 ? lo * c[r - 1] : 0.0);
        c[r] = up / den;
        x[r] = (x[r] - (r > 0 ? lo * x[r - 1] : 0.0)) / den;
    }
    for (int r = m - 2; r >= 0; r--) x[r] -= c[r] * x[r + 1];
    free(c);
}

int ora_spline_ypp(int n, double dt, const double *Et, double *ypp) {
    nak_sys S;
    if (nak_build(n, dt, &S)) return -1;
    int m = n - 2;
    double *x = ypp + 1;
    for (int r = 1; r <= n - 2; r++) {
        double hm = knot(r, dt) - knot(r - 1, dt), hp = knot(r + 1, dt) - knot(r, dt);
        x[r - 1] = (Et[r + 1] - Et[r]) / hp - (Et[r] - Et[r - 1]) / hm;
    }
    nak_thomas(&S, x, 0);
    ypp[0] = S.e0a * ypp[1] + S.e0b * ypp[2];
    ypp[n - 1] = S.e1a * ypp[n - 2] + S.e1b * ypp[n - 3];
    (void)m;
    nak_free(&S);
    return 0;
}

/* Interval l with t_l <= t <= t_{l+1}, clamped to [0, n-2]. */
static int spline_interval(int n, double dt, double t) {
    int l = (int)floor(t / dt);
    if (l < 0) l = 0;
    if (l > n - 2) l = n - 2;
    while (l > 0 && t < knot(l, dt)) l--;
    while (l < n - 2 && t > knot(l + 1, dt)) l++;
    return l;
}

/* Value coefficients of the cubic on interval l at offset s = t - t_l:
 * S(t) = cyl*y_l + cyr*y_r + cpl*ypp_l + cpr*ypp_r. */
static void spline_coefs(double s, double hh, double *cyl, double *cyr, double *cpl, double *cpr) {
    *cyl = 1.0 - s / hh;
    *cyr = s / hh;
    *cpl = -s * hh / 3.0 + 0.5 * s * s - s * s * s / (6.0 * hh);
    *cpr = -s * hh / 6.0 + s * s * s / (6.0 * hh);
}

double ora_spline_val(int n, double dt, const double *Et, const double *ypp, double t) {
    int l = spline_interval(n, dt, t), r = l + 1;
    double s = t - knot(l, dt), hh = knot(r, dt) - knot(l, dt);
    /* nested form of the cubic (de Boor's Taylor expansion about t_l) */
    return Et[l] + s * ((Et[r] - Et[l]) / hh - (ypp[r] / 6.0 + ypp[l] / 3.0) * hh
                        + s * (0.5 * ypp[l] + s * ((ypp[r] - ypp[l]) / (6.0 * hh))));
}

/* Adds Phi^T g to gE, where Phi maps samples Et[0..n) to the spline values at
 * t = (l + frac)*dt, l = 0..n-2 (the discrete transpose of ora_spline_ypp +
 * ora_spline_val). */
static int spline_transpose(int n, double dt, double frac, const double *g, double *gE) {
    nak_sys S;
    if (n < 4 || nak_build(n, dt, &S)) return -1;
    int m = n - 2;
    double *gp = (double *)calloc((size_t)n, sizeof(double));
    for (int l = 0; l < n - 1; l++) {
        double t = ((double)l + frac) * dt;
        double s = t - knot(l, dt), hh = knot(l + 1, dt) - knot(l, dt);
        double a, b, c, d;
        spline_coefs(s, hh, &a, &b, &c, &d);
        gE[l] += a * g[l];
        gE[l + 1] += b * g[l];
        gp[l] += c * g[l];
        gp[l + 1] += d * g[l];
    }
    double *x = (double *)malloc((size_t)m * sizeof(double));
    for (int r = 0; r < m; r++) x[r] = gp[r + 1];
    x[0] += S.e0a * gp[0];
    x[1] += S.e0b * gp[0];
    x[m - 1] += S.e1a * gp[n - 1];
    x[m - 2] += S.e1b * gp[n - 1];
    nak_thomas(&S, x, 1);
    for (int r = 1; r <= n - 2; r++) {
        double hm = knot(r, dt) - knot(r - 1, dt), hp = knot(r + 1, dt) - knot(r, dt);
        double gb = x[r - 1];
        gE[r + 1] += gb / hp;
        gE[r] -= gb / hp + gb / hm;
        gE[r - 1] += gb / hm;
    }
    free(x);
    free(gp);
    nak_free(&S);
    return 0;
}

/* ------------------------------------------------------------- RK4 sweep */

typedef struct {
    int n3;
    double *f, *U, *Ut, *d;
} rk4_work;

static void rk4_alloc(rk4_work *W, int n3) {
    W->n3 = n3;
    W->f = (double *)malloc((size_t)n3 * sizeof(double));
    W->U = (double *)malloc((size_t)n3 * sizeof(double));
    W->Ut = (double *)malloc((size_t)n3 * sizeof(double));
    W->d = (double *)malloc((size_t)n3 * sizeof(double));
}

static void rk4_release(rk4_work *W) {
    free(W->f);
    free(W->U);
    free(W->Ut);
    free(W->d);
}

/* One classical RK4 step in place; stage algebra of cu-F:459-562 with the
 * E sources of cu-F:766-793 (E0 = Et[i], Eh = spline at (i+1/2)dt,
 * E1 = Et[i+1]). */
static void rk4_step(const ora_params *P, int nrows, int ncols, double dt, double *y,
                     const double *gh, double E0, double Eh, double E1, rk4_work *W) {
    const int n3 = W->n3;
    double *f = W->f, *U = W->U, *Ut = W->Ut, *d = W->d;
    ora_rhs(P, nrows, ncols, y, gh, E0, f);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n3; k++) {
        U[k] = y[k] + dt * 0.5 * f[k];
        d[k] = 1.0 / 6.0 * dt * f[k];
    }
    ora_rhs(P, nrows, ncols, U, gh, Eh, f);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n3; k++) {
        Ut[k] = y[k] + dt * 0.5 * f[k];
        d[k] = d[k] + 1.0 / 3.0 * dt * f[k];
    }
    ora_rhs(P, nrows, ncols, Ut, gh, Eh, f);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n3; k++) {
        U[k] = y[k] + dt * 1.0 * f[k];
        d[k] = d[k] + 1.0 / 3.0 * dt * f[k];
    }
    ora_rhs(P, nrows, ncols, U, gh, E1, f);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n3; k++) y[k] = y[k] + d[k] + dt * 1.0 / 6.0 * f[k];
}

int ora_forward(const ora_params *P, double dt, const double *Et, int nt,
                int nrows, int ncols, const double *y0, const double *gh,
                int nstep, int ns, double *ys, double *yf) {
    const int n = nrows * ncols, n3 = 3 * n;
    double *ypp = (double *)malloc((size_t)(nt + 1) * sizeof(double));
    if (ora_spline_ypp(nt + 1, dt, Et, ypp)) {
        free(ypp);
        return -1;
    }
    double *y = (double *)malloc((size_t)n3 * sizeof(double));
    memcpy(y, y0, (size_t)n3 * sizeof(double));
    rk4_work W;
    rk4_alloc(&W, n3);
    for (int i = 0; i < nt; i++) {
        double Eh = ora_spline_val(nt + 1, dt, Et, ypp, (i + 0.5) * dt);
        rk4_step(P, nrows, ncols, dt, y, gh, Et[i], Eh, Et[i + 1], &W);
        if (nstep > 0 && (i + 1) % nstep == 0) {
            int ks = (i + 1) / nstep - 1;
            if (ks < ns) memcpy(ys + (size_t)ks * n3, y, (size_t)n3 * sizeof(double));
        }
    }
    memcpy(yf, y, (size_t)n3 * sizeof(double));
    rk4_release(&W);
    free(y);
    free(ypp);
    return 0;
}

/* -------------------------------------------------------------- objective */

int ora_objective_eval(const ora_objective *obj, const int *active_index, int n,
                       const double *yT, double *L0, double *zT) {
    const int nn = obj->n_num;
    double *yc = (double *)malloc((size_t)nn * sizeof(double));
    double *zc = (double *)malloc((size_t)nn * sizeof(double));
    double acc = 0.0;
    int nact = 0;
    for (int k = 0; k < n; k++) nact += active_index[k] > 0;
    if (nact != nn) {
        free(yc);
        free(zc);
        return -2;
    }
    for (int c = 0; c < 3; c++) {
        for (int k = 0; k < n; k++)
            if (active_index[k] > 0) yc[active_index[k] - 1] = yT[(size_t)c * n + k];
        /* z = S*y in CSC column order (cu-G:1514-1522), then z *= -gamma */
        for (int r = 0; r < nn; r++) zc[r] = 0.0;
        for (int col = 0; col < nn; col++)
            for (int64_t q = obj->Jc[col]; q < obj->Jc[col + 1]; q++)
                zc[obj->Ir[q]] += obj->Sv[q] * yc[col];
        double gg = -obj->gamma[c];
        for (int r = 0; r < nn; r++) zc[r] *= gg;
        double dot = 0.0;
        for (int r = 0; r < nn; r++) dot += yc[r] * zc[r];
        acc -= dot;
        for (int k = 0; k < n; k++)
            zT[(size_t)c * n + k] = active_index[k] > 0 ? zc[active_index[k] - 1] : NAN;
    }
    *L0 = acc;
    free(yc);
    free(zc);
    return 0;
}

/* sum_k a[k]*b[k] over non-NaN products, in the reference's order: 16x16
 * blocks in block-row-major order, row-major inside a block (cu-G:1457-1483
 * summed by vec_sum, cu-G:1553-1561). */
static double nan_dot_blocked(const double *a, const double *b, int nrows, int ncols) {
    double total = 0.0;
    for (int bi = 0; bi < nrows; bi += 16)
        for (int bj = 0; bj < ncols; bj += 16) {
            double part = 0.0;
            for (int i = bi; i < bi + 16 && i < nrows; i++)
                for (int j = bj; j < bj + 16 && j < ncols; j++) {
                    double t = a[i * ncols + j] * b[i * ncols + j];
                    if (!isnan(t)) part += t;
                }
            total += part;
        }
    return total;
}

static double dot_plain(const double *a, const double *b, int n) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

/* ------------------------------------------------- reference-mode adjoint */

/* Cubic Hermite weights at t = 1/3 and the partial quartic weights at 1/2
 * used to rebuild the forward state at the step midpoint (cu-G:1217-1241,
 * 1295-1298). */
static void hermite_weights(double h3[4], double h4[4], double *c2) {
    double t = 1.0 / 3.0;
    h3[0] = (t - 1.0) * (t - 1.0) * (2.0 * t + 1.0);
    h3[1] = t * (t - 1.0) * (t - 1.0);
    h3[2] = t * t * (3.0 - 2.0 * t);
    h3[3] = t * t * (t - 1.0);
    t = 1.0 / 2.0;
    h4[0] = ((1.0 + 2.0 * t + 9.0 * t * t) * (t - 1.0) * (t - 1.0));
    h4[1] = (t * (t - 1.0) * (t - 1.0));
    h4[2] = (-t * t * (6.0 - 16.0 * t + 9.0 * t * t));
    h4[3] = ((t - 1.0) * (9.0 * t - 5.0) * t * t / 4.0);
    *c2 = (27.0 * t * t * (t - 1.0) * (t - 1.0) / 4.0);
}

int ora_grad_ref(const ora_params *P, double dt, const double *Et, int nt,
                 int nrows, int ncols, const double *y0, const double *gh,
                 const int *active_index, const ora_objective *obj, double alpha,
                 double *gradE, double *L0, double *LE, double *Lcost, double *yf) {
    const int n = nrows * ncols, n3 = 3 * n;
    double *ypp = (double *)malloc((size_t)(nt + 1) * sizeof(double));
    if (ora_spline_ypp(nt + 1, dt, Et, ypp)) {
        free(ypp);
        return -1;
    }
    double *yt = (double *)malloc((size_t)(nt + 1) * n3 * sizeof(double));
    if (!yt) {
        free(ypp);
        return -3;
    }
    memcpy(yt, y0, (size_t)n3 * sizeof(double));
    rk4_work W;
    rk4_alloc(&W, n3);
    for (int i = 0; i < nt; i++) {
        double *y = yt + (size_t)(i + 1) * n3;
        memcpy(y, yt + (size_t)i * n3, (size_t)n3 * sizeof(double));
        double Eh = ora_spline_val(nt + 1, dt, Et, ypp, (i + 0.5) * dt);
        rk4_step(P, nrows, ncols, dt, y, gh, Et[i], Eh, Et[i + 1], &W);
    }
    rk4_release(&W);
    if (yf) memcpy(yf, yt + (size_t)nt * n3, (size_t)n3 * sizeof(double));

    double *z = (double *)malloc((size_t)n3 * sizeof(double));
    int rc = ora_objective_eval(obj, active_index, n, yt + (size_t)nt * n3, L0, z);
    if (rc) {
        free(z);
        free(yt);
        free(ypp);
        return rc;
    }
    *LE = dt * dot_plain(Et, Et, nt + 1);
    *Lcost = 0.5 * (*L0) + 0.5 * alpha * (*LE);

    double *zgh = (double *)malloc((size_t)(nt + 1) * sizeof(double));
    zgh[nt] = nan_dot_blocked(z, gh, nrows, ncols);

    double h3[4], h4[4], c2;
    hermite_weights(h3, h4, &c2);
    double *m0 = (double *)malloc((size_t)n3 * sizeof(double));
    double *m1 = (double *)malloc((size_t)n3 * sizeof(double));
    double *y3 = (double *)malloc((size_t)n3 * sizeof(double));
    double *yh = (double *)malloc((size_t)n3 * sizeof(double));
    double *Z = (double *)malloc((size_t)n3 * sizeof(double));
    double *Zt = (double *)malloc((size_t)n3 * sizeof(double));
    double *dz = (double *)malloc((size_t)n3 * sizeof(double));
    double *fz = (double *)malloc((size_t)n3 * sizeof(double));
    for (int i = nt; i > 0; i--) {
        const double *yi = yt + (size_t)i * n3;        /* y(t_i)     */
        const double *yim = yt + (size_t)(i - 1) * n3; /* y(t_{i-1}) */
        /* midpoint reconstruction (cu-G:1244-1301, order of cu-G:1874-1881) */
        ora_rhs(P, nrows, ncols, yim, gh, Et[i - 1], m0);
        ora_rhs(P, nrows, ncols, yi, gh, Et[i], m1);
#pragma omp parallel for schedule(static)
        for (int k = 0; k < n3; k++) {
            double a0 = m0[k] * dt, a1 = m1[k] * dt;
            y3[k] = h3[0] * yim[k] + h3[1] * a0 + h3[2] * yi[k] + h3[3] * a1;
            yh[k] = h4[0] * yim[k] + h4[1] * a0 + h4[2] * yi[k] + h4[3] * a1;
        }
        double E3 = ora_spline_val(nt + 1, dt, Et, ypp, (i - 1 + 1.0 / 3.0) * dt);
        ora_rhs(P, nrows, ncols, y3, gh, E3, m0);
#pragma omp parallel for schedule(static)
        for (int k = 0; k < n3; k++) yh[k] = yh[k] + c2 * (m0[k] * dt);
        /* backward RK4 stages (cu-G:1349-1427, order of cu-G:1885-1891) */
        ora_adj_rhs(P, nrows, ncols, z, yi, fz);
#pragma omp parallel for schedule(static)
        for (int k = 0; k < n3; k++) {
            Z[k] = z[k] + 0.5 * dt * fz[k];
            dz[k] = 1.0 / 6.0 * dt * fz[k];
        }
        ora_adj_rhs(P, nrows, ncols, Z, yh, fz);
#pragma omp parallel for schedule(static)
        for (int k = 0; k < n3; k++) {
            Zt[k] = z[k] + 0.5 * dt * fz[k];
            dz[k] = dz[k] + 2.0 / 6.0 * dt * fz[k];
        }
        ora_adj_rhs(P, nrows, ncols, Zt, yh, fz);
#pragma omp parallel for schedule(static)
        for (int k = 0; k < n3; k++) {
            Z[k] = z[k] + dt * fz[k];
            dz[k] = dz[k] + 2.0 / 6.0 * dt * fz[k];
        }
        ora_adj_rhs(P, nrows, ncols, Z, yim, fz);
#pragma omp parallel for schedule(static)
        for (int k = 0; k < n3; k++) z[k] = z[k] + dz[k] + 1.0 / 6.0 * dt * fz[k];
        zgh[i - 1] = nan_dot_blocked(z, gh, nrows, ncols);
    }
    for (int i = 0; i < nt + 1; i++) gradE[i] = alpha * Et[i] - zgh[i];

    free(m0); free(m1); free(y3); free(yh); free(Z); free(Zt); free(dz); free(fz);
    free(zgh); free(z); free(yt); free(ypp);
    return 0;
}

/* ------------------------------------------------------ exact-mode adjoint */

/* sum over active cells of gh * a_u (the E-source direction b^T a). */
static double b_dot(const double *a, const double *gh, int n) {
    double s = 0.0;
    for (int k = 0; k < n; k++)
        if (!isnan(gh[k])) s += gh[k] * a[k];
    return s;
}

int ora_grad_exact(const ora_params *P, double dt, const double *Et, int nt,
                   int nrows, int ncols, const double *y0, const double *gh,
                   const int *active_index, const ora_objective *obj, double alpha,
                   double *gradE, double *L0, double *LE, double *Lcost, double *yf) {
    const int n = nrows * ncols, n3 = 3 * n;
    double *ypp = (double *)malloc((size_t)(nt + 1) * sizeof(double));
    if (ora_spline_ypp(nt + 1, dt, Et, ypp)) {
        free(ypp);
        return -1;
    }
    double *Eh = (double *)malloc((size_t)nt * sizeof(double));
    for (int i = 0; i < nt; i++) Eh[i] = ora_spline_val(nt + 1, dt, Et, ypp, (i + 0.5) * dt);
    double *yt = (double *)malloc((size_t)(nt + 1) * n3 * sizeof(double));
    if (!yt) {
        free(Eh);
        free(ypp);
        return -3;
    }
    memcpy(yt, y0, (size_t)n3 * sizeof(double));
    rk4_work W;
    rk4_alloc(&W, n3);
    for (int i = 0; i < nt; i++) {
        double *y = yt + (size_t)(i + 1) * n3;
        memcpy(y, yt + (size_t)i * n3, (size_t)n3 * sizeof(double));
        rk4_step(P, nrows, ncols, dt, y, gh, Et[i], Eh[i], Et[i + 1], &W);
    }
    rk4_release(&W);
    if (yf) memcpy(yf, yt + (size_t)nt * n3, (size_t)n3 * sizeof(double));

    double *lam = (double *)malloc((size_t)n3 * sizeof(double));
    int rc = ora_objective_eval(obj, active_index, n, yt + (size_t)nt * n3, L0, lam);
    if (rc) {
        free(lam); free(yt); free(Eh); free(ypp);
        return rc;
    }
    for (int k = 0; k < n3; k++) lam[k] = -lam[k]; /* lambda_T = dJ/dy = -z */
    *LE = dt * dot_plain(Et, Et, nt + 1);
    *Lcost = 0.5 * (*L0) + 0.5 * alpha * (*LE);

    double *gE = (double *)calloc((size_t)(nt + 1), sizeof(double));
    double *gEh = (double *)calloc((size_t)nt, sizeof(double));
    double *k1 = (double *)malloc((size_t)n3 * sizeof(double));
    double *Y2 = (double *)malloc((size_t)n3 * sizeof(double));
    double *Y3 = (double *)malloc((size_t)n3 * sizeof(double));
    double *Y4 = (double *)malloc((size_t)n3 * sizeof(double));
    double *a = (double *)malloc((size_t)n3 * sizeof(double));
    double *mu = (double *)malloc((size_t)n3 * sizeof(double));
    double *acc = (double *)malloc((size_t)n3 * sizeof(double));
    for (int s = nt - 1; s >= 0; s--) {
        const double *y = yt + (size_t)s * n3;
        /* recompute the stage states of step s */
        ora_rhs(P, nrows, ncols, y, gh, Et[s], k1);
        for (int k = 0; k < n3; k++) Y2[k] = y[k] + dt * 0.5 * k1[k];
        ora_rhs(P, nrows, ncols, Y2, gh, Eh[s], k1);
        for (int k = 0; k < n3; k++) Y3[k] = y[k] + dt * 0.5 * k1[k];
        ora_rhs(P, nrows, ncols, Y3, gh, Eh[s], k1);
        for (int k = 0; k < n3; k++) Y4[k] = y[k] + dt * 1.0 * k1[k];
        /* transposed stages: a_s is the adjoint of k_s, mu_s = f_y(Y_s)^T a_s */
        for (int k = 0; k < n3; k++) a[k] = dt / 6.0 * lam[k];
        gE[s + 1] += b_dot(a, gh, n);
        ora_adj_rhs(P, nrows, ncols, a, Y4, mu);
        for (int k = 0; k < n3; k++) {
            acc[k] = mu[k];
            a[k] = dt / 3.0 * lam[k] + dt * mu[k];
        }
        double gh_sum = b_dot(a, gh, n);
        ora_adj_rhs(P, nrows, ncols, a, Y3, mu);
        for (int k = 0; k < n3; k++) {
            acc[k] += mu[k];
            a[k] = dt / 3.0 * lam[k] + dt * 0.5 * mu[k];
        }
        gh_sum += b_dot(a, gh, n);
        gEh[s] += gh_sum;
        ora_adj_rhs(P, nrows, ncols, a, Y2, mu);
        for (int k = 0; k < n3; k++) {
            acc[k] += mu[k];
            a[k] = dt / 6.0 * lam[k] + dt * 0.5 * mu[k];
        }
        gE[s] += b_dot(a, gh, n);
        ora_adj_rhs(P, nrows, ncols, a, y, mu);
        for (int k = 0; k < n3; k++) lam[k] = lam[k] + (acc[k] + mu[k]);
    }
    spline_transpose(nt + 1, dt, 0.5, gEh, gE);
    for (int i = 0; i < nt + 1; i++) gradE[i] = (gE[i] + alpha * dt * Et[i]) / dt;

    free(k1); free(Y2); free(Y3); free(Y4); free(a); free(mu); free(acc);
    free(gE); free(gEh); free(lam); free(yt); free(Eh); free(ypp);
    return 0;
}
