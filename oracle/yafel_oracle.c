/*
 * yafel_oracle.c -- CPU restatement of the reference's CG-FEM assemble + solve
 * path.  TEST INFRASTRUCTURE ONLY (the checker): imported by tests/, by the
 * smoke check and by the bench's CPU-baseline leg, never by the product.
 *
 * Citations are file:line in the YAFEL source tree.  The restatement follows the
 * reference's arithmetic order where that matters for the integer results
 * (dof numbering, sparsity patterns) and states the published algorithm
 * otherwise.  Built with -ffp-contract=off so results do not depend on FMA
 * contraction.
 */
#include "yafel_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_MAX_NEN 125
#define OR_MAX_NQ 216

int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ===================================================================== */
/* Quadrature                                                              */
/* ===================================================================== */

/* Gauss-Legendre points by Newton iteration on P_n, tolerance 1e-15 on |P_n|
 * (src/quadrature/QuadratureRule.cpp:66-106). */
void or_gauss_legendre_1d(int n, double *x, double *w) {
    const double PI = atan2(1., 1.) * 4;
    for (int i = 0; i < n; ++i) {
        double xx = -cos(PI * (1 + i - 0.25) / (n + 0.5));
        double Pold, Pn, Pnew, dP;
        int guard = 0;
        do {
            Pold = 1;
            Pn = xx;
            for (int k = 2; k <= n; ++k) {
                Pnew = ((2 * k - 1) * xx * Pn - (k - 1) * Pold) / k;
                Pold = Pn;
                Pn = Pnew;
            }
            dP = (n / (xx * xx - 1)) * (xx * Pn - Pold);
            xx -= Pn / dP;
        } while (fabs(Pn) > 1.0e-15 && ++guard < 200);
        x[i] = xx;
        w[i] = 2.0 / ((1 - xx * xx) * (dP * dP));
    }
}

/* Gauss-Lobatto points: Newton-type fixed point x <- x - (x - P_{n-2}/P_{n-1})/n
 * started from Chebyshev-Lobatto points (src/quadrature/QuadratureRule.cpp:25-63). */
void or_gauss_lobatto_1d(int n, double *x, double *w) {
    const double PI = atan2(1., 1.) * 4;
    for (int i = 0; i < n; ++i) {
        double xx = -cos((PI * i) / (n - 1));
        double xold, Pold, Pn, Pnew;
        int guard = 0;
        do {
            xold = xx;
            Pold = 1;
            Pn = xx;
            for (int k = 2; k < n; ++k) {
                Pnew = ((2 * k - 1) * xx * Pn - (k - 1) * Pold) / k;
                Pold = Pn;
                Pn = Pnew;
            }
            xx = xx - (xx - Pold / Pn) / n;
        } while (fabs(xx - xold) > 1.0e-15 && ++guard < 200);
        x[i] = xx;
        w[i] = 2 / (n * (n - 1) * Pn * Pn);
    }
}

/* Tensor-product rule integrating polynomials of degree `order` exactly,
 * x fastest (src/quadrature/QuadratureRule.cpp:109-175). pts is nq*3. */
int or_tensor_rule(int lobatto, int dim, int order, double *pts, double *w) {
    if (dim == 0) {
        pts[0] = pts[1] = pts[2] = 0;
        w[0] = 1;
        return 1;
    }
    double x1[32], w1[32];
    int n;
    if (!lobatto) {
        n = (order + 1) / 2 + (order + 1) % 2;
        or_gauss_legendre_1d(n, x1, w1);
    } else {
        n = (order + 3) / 2 + (order + 3) % 2;
        or_gauss_lobatto_1d(n, x1, w1);
    }
    int q = 0;
    if (dim == 1) {
        for (int i = 0; i < n; ++i) {
            pts[3 * q] = x1[i]; pts[3 * q + 1] = 0; pts[3 * q + 2] = 0;
            w[q++] = w1[i];
        }
    } else if (dim == 2) {
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                pts[3 * q] = x1[j]; pts[3 * q + 1] = x1[i]; pts[3 * q + 2] = 0;
                w[q++] = w1[i] * w1[j];
            }
    } else {
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                for (int k = 0; k < n; ++k) {
                    pts[3 * q] = x1[k]; pts[3 * q + 1] = x1[j]; pts[3 * q + 2] = x1[i];
                    w[q++] = w1[i] * w1[j] * w1[k];
                }
    }
    return q;
}

int or_triangle_rule_collapsed(int order, double *pts, double *w);

/* Triangle rule on the unit right triangle (0,0),(1,0),(0,1), exact for degree
 * `order`.  The reference tabulates Dunavant-type rules
 * (src/quadrature/TriangleQuadratureRules.cpp:9-221); the oracle uses an
 * independent rule of the same exactness (Gauss-Legendre on the collapsed
 * square, x = u(1-v), y = v, Jacobian 1-v), so the assembled values agree up to
 * rounding while the product's tables are checked, not copied. */
/* Optional override with the reference's own tabulated rules (installed by
 * oracle.py from the fixture that tests/golden/make_golden.py generated by
 * running src/quadrature/TriangleQuadratureRules.cpp). */
static int g_tri_n[16];
static double g_tri_pts[16][3 * 64], g_tri_w[16][64];
void or_set_triangle_rule(int order, const double *pts, const double *w, int n) {
    if (order < 0 || order >= 16 || n > 64) return;
    g_tri_n[order] = n;
    memcpy(g_tri_pts[order], pts, sizeof(double) * 3 * n);
    memcpy(g_tri_w[order], w, sizeof(double) * n);
}

int or_triangle_rule(int order, double *pts, double *w) {
    if (order >= 0 && order < 16 && g_tri_n[order] > 0) {
        memcpy(pts, g_tri_pts[order], sizeof(double) * 3 * g_tri_n[order]);
        memcpy(w, g_tri_w[order], sizeof(double) * g_tri_n[order]);
        return g_tri_n[order];
    }
    return or_triangle_rule_collapsed(order, pts, w);
}

int or_triangle_rule_collapsed(int order, double *pts, double *w) {
    int n = (order + 3) / 2; /* ceil((order+2)/2) */
    double x1[32], w1[32];
    or_gauss_legendre_1d(n, x1, w1);
    int q = 0;
    for (int i = 0; i < n; ++i) {
        double v = 0.5 * (x1[i] + 1), wv = 0.5 * w1[i];
        for (int j = 0; j < n; ++j) {
            double u = 0.5 * (x1[j] + 1), wu = 0.5 * w1[j];
            pts[3 * q] = u * (1 - v);
            pts[3 * q + 1] = v;
            pts[3 * q + 2] = 0;
            w[q++] = wu * wv * (1 - v);
        }
    }
    return q;
}

/* ===================================================================== */
/* Polynomials, dual numbers, dense LU                                     */
/* ===================================================================== */

typedef struct { double f, d; } dual;
static dual dmk(double f, double d) { dual r = {f, d}; return r; }
static dual dadd(dual a, dual b) { return dmk(a.f + b.f, a.d + b.d); }
static dual dsub(dual a, dual b) { return dmk(a.f - b.f, a.d - b.d); }
static dual dmul(dual a, dual b) { return dmk(a.f * b.f, a.d * b.f + a.f * b.d); }
static dual ddiv(dual a, dual b) { return dmk(a.f / b.f, (a.d * b.f - a.f * b.d) / (b.f * b.f)); }
static dual dscale(double s, dual a) { return dmk(s * a.f, s * a.d); }
/* pow of a dual with integer exponent, as include/utils/DualNumber.hpp:162-166 */
static dual dpowi(dual x, int e) { return dmk(pow(x.f, e), x.d * e * pow(x.f, e - 1)); }

/* Jacobi polynomial P_n^{(alpha,beta)} coefficients, highest degree first, by
 * the three-term recurrence (src/element/ShapeFunctionUtils.cpp:16-62). */
static int jacobi_coeffs(int n, double alpha, double beta, double *out) {
    double c1[32], c2[32], c[32];
    int n1 = 2, n2 = 1, nc;
    c1[0] = (alpha + beta + 2) / 2;
    c1[1] = (alpha - beta) / 2;
    c2[0] = 1.0;
    if (n == 0) { out[0] = 1.0; return 1; }
    if (n == 1) { out[0] = c1[0]; out[1] = c1[1]; return 2; }
    memcpy(c, c1, sizeof(double) * 2);
    nc = 2;
    for (int i = 1; i < n; ++i) {
        double tmp = i + alpha + beta + 1;
        double a = (2 * i + alpha + beta + 1) * (2 * i + alpha + beta + 2) / (2 * (i + 1) * tmp);
        double b = (beta * beta - alpha * alpha) * (2 * i + alpha + beta + 1) /
                   (2 * (i + 1) * tmp * (2 * i + alpha + beta));
        double cc = (i + alpha) * (i + beta) * (2 * i + alpha + beta + 2) /
                    ((i + 1) * tmp * (2 * i + alpha + beta));
        c[nc++] = 0;
        for (int k = 0; k < nc; ++k) c[k] *= a;
        for (int k = 0; k < n1; ++k) c[nc - 1 - k] -= b * c1[n1 - 1 - k];
        for (int k = 0; k < n2; ++k) c[nc - 1 - k] -= cc * c2[n2 - 1 - k];
        memcpy(c2, c1, sizeof(double) * n1); n2 = n1;
        memcpy(c1, c, sizeof(double) * nc); n1 = nc;
    }
    memcpy(out, c, sizeof(double) * nc);
    return nc;
}

/* Horner evaluation (include/element/ShapeFunctionUtils.hpp:48-57). */
static double poly_eval(const double *c, int nc, double x) {
    double r = 0;
    for (int i = 0; i < nc; ++i) { r *= x; r += c[i]; }
    return r;
}
static dual poly_eval_d(const double *c, int nc, dual x) {
    dual r = dmk(0, 0);
    for (int i = 0; i < nc; ++i) { r = dmul(r, x); r = dadd(r, dmk(c[i], 0)); }
    return r;
}

/* LU with partial (row) pivoting, Golub & Van Loan Alg. 3.4.1.  A is n*n
 * row-major, overwritten by L\U; piv records the row permutation. */
static void lu_factor(double *A, int n, int *piv) {
    for (int i = 0; i < n; ++i) piv[i] = i;
    for (int k = 0; k < n; ++k) {
        int p = k;
        double best = fabs(A[k * n + k]);
        for (int i = k + 1; i < n; ++i)
            if (fabs(A[i * n + k]) > best) { best = fabs(A[i * n + k]); p = i; }
        if (p != k) {
            for (int j = 0; j < n; ++j) { double t = A[k * n + j]; A[k * n + j] = A[p * n + j]; A[p * n + j] = t; }
            int t = piv[k]; piv[k] = piv[p]; piv[p] = t;
        }
        for (int i = k + 1; i < n; ++i) {
            A[i * n + k] /= A[k * n + k];
            double m = A[i * n + k];
            for (int j = k + 1; j < n; ++j) A[i * n + j] -= m * A[k * n + j];
        }
    }
}
static void lu_solve(const double *LU, int n, const int *piv, const double *b, double *x) {
    double y[OR_MAX_NEN];
    for (int i = 0; i < n; ++i) {
        double s = b[piv[i]];
        for (int j = 0; j < i; ++j) s -= LU[i * n + j] * y[j];
        y[i] = s;
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = y[i];
        for (int j = i + 1; j < n; ++j) s -= LU[i * n + j] * x[j];
        x[i] = s / LU[i * n + i];
    }
}

/* ===================================================================== */
/* Reference elements                                                      */
/* ===================================================================== */

static double snap_to(double x, double s) { return round(x / s) * s; }

/* Local (reference-element) nodes.  Tensor product: GLL points, x fastest
 * (src/element/make_tensorproduct_element.cpp:17-31,148-193).  Triangle:
 * Blyth-Pozrikidis points from the GLL points, snapped to 2^-21
 * (src/element/make_simplex_element.cpp:17-26,94-97,156-176). */
int or_local_nodes(int topology, int dim, int p, double *pts) {
    int n = p + 1;
    double l[32], lw[32];
    or_gauss_lobatto_1d(n, l, lw);
    int idx = 0;
    if (topology == OR_TENSOR || dim == 1) {
        if (dim == 1) {
            for (int i = 0; i < n; ++i) { pts[3 * idx] = l[i]; pts[3 * idx + 1] = 0; pts[3 * idx + 2] = 0; ++idx; }
        } else if (dim == 2) {
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j) { pts[3 * idx] = l[j]; pts[3 * idx + 1] = l[i]; pts[3 * idx + 2] = 0; ++idx; }
        } else if (dim == 3) {
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j)
                    for (int k = 0; k < n; ++k) {
                        pts[3 * idx] = l[k]; pts[3 * idx + 1] = l[j]; pts[3 * idx + 2] = l[i]; ++idx;
                    }
        }
        return idx;
    }
    if (topology == OR_SIMPLEX && dim == 2) {
        const double snap = 1.0 / (2 << 20);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n - i; ++j) {
                int k = n - i - j - 1;
                double vi = (l[i] + 1) / 2, vj = (l[j] + 1) / 2, vk = (l[k] + 1) / 2;
                pts[3 * idx] = snap_to((1 + 2 * vj - vi - vk) / 3, snap);
                pts[3 * idx + 1] = snap_to((1 + 2 * vi - vj - vk) / 3, snap);
                pts[3 * idx + 2] = snap_to(0.0, snap);
                ++idx;
            }
        return idx;
    }
    return 0; /* tetrahedra are not part of the restated path */
}

/* Volume rule of an element: GL tensor rule of order 2p for tensor products
 * (make_tensorproduct_element.cpp:127-128), a degree-2p triangle rule for
 * triangles (make_simplex_element.cpp:99-100). */
int or_element_rule(int topology, int dim, int p, double *pts, double *w) {
    if (topology == OR_TENSOR || dim == 1) return or_tensor_rule(0, dim, 2 * p, pts, w);
    if (topology == OR_SIMPLEX && dim == 2) return or_triangle_rule(2 * p > 1 ? 2 * p : 1, pts, w);
    return 0;
}

/* Nodal shape functions and reference gradients at the given points, via the
 * Vandermonde matrix of an orthogonal basis, V(i,j)=phi_j(x_i), solved as
 * V^T N = phi(xi) with partial-pivot LU; gradients by forward-mode dual
 * numbers.  Tensor product: Legendre products
 * (src/element/ShapeFunctionUtils.cpp:64-143).  Triangle: Koornwinder basis on
 * the node set with the top vertex moved to y=0.999999999
 * (src/element/ShapeFunctionUtils.cpp:145-217). N is nq*nen, dN nq*nen*dim. */
int or_shape_functions(int topology, int dim, int p, const double *qpts, int nq,
                       double *N, double *dN) {
    double nodes[3 * OR_MAX_NEN];
    int nen = or_local_nodes(topology, dim, p, nodes);
    if (nen <= 0 || nen > OR_MAX_NEN) return -1;
    double *V = (double *)malloc(sizeof(double) * OR_MAX_NEN * OR_MAX_NEN);
    double VT[OR_MAX_NEN * OR_MAX_NEN];
    int piv[OR_MAX_NEN];
    double coef[32][32];
    int ncoef[32];
    int tri = (topology == OR_SIMPLEX && dim == 2);
    int mm[OR_MAX_NEN];
    double jac2[OR_MAX_NEN][32];
    int njac2[OR_MAX_NEN];
    int np1 = p + 1;
    for (int k = 0; k < np1; ++k) ncoef[k] = jacobi_coeffs(k, 0, 0, coef[k]);
    if (tri) {
        int c = 0;
        for (int i = 0; i <= p; ++i)
            for (int j = 0; j <= p; ++j)
                if (i + j <= p) { mm[c] = i; njac2[c] = jacobi_coeffs(j, 2 * i + 1, 0, jac2[c]); ++c; }
        for (int i = 0; i < nen; ++i) if (nodes[3 * i + 1] > .999999999) nodes[3 * i + 1] = .999999999;
    }
    /* basis evaluation with dual numbers: grad direction g (-1 = value only) */
    #define BASIS(jj, X, g, outv)                                                         \
    do {                                                                                   \
        dual xd[3];                                                                        \
        for (int di = 0; di < 3; ++di) xd[di] = dmk((X)[di], (g) == di ? 1.0 : 0.0);       \
        if (!tri) {                                                                        \
            int pp = np1;                                                                  \
            dual bv_;                                                                      \
            if (dim == 1) bv_ = poly_eval_d(coef[jj], ncoef[jj], xd[0]);                     \
            else if (dim == 2) {                                                           \
                int ii = (jj) / pp, kk = (jj) % pp;                                        \
                bv_ = dmul(poly_eval_d(coef[kk], ncoef[kk], xd[0]),                        \
                         poly_eval_d(coef[ii], ncoef[ii], xd[1]));                         \
            } else {                                                                       \
                int ii = (jj) / (pp * pp), kk2 = ((jj) % (pp * pp)) / pp, kk = (jj) % pp;  \
                bv_ = dmul(dmul(poly_eval_d(coef[kk], ncoef[kk], xd[0]),                   \
                              poly_eval_d(coef[kk2], ncoef[kk2], xd[1])),                  \
                         poly_eval_d(coef[ii], ncoef[ii], xd[2]));                         \
            }                                                                              \
            outv = bv_;                                                                    \
        } else {                                                                           \
            int m_ = mm[jj];                                                               \
            dual r = dsub(ddiv(dmul(dmk(2, 0), dadd(dmk(1, 0), xd[0])),                    \
                               dsub(dmk(1, 0), xd[1])), dmk(1, 0));                        \
            dual s = xd[1];                                                                \
            dual hs = ddiv(dsub(dmk(1, 0), s), dmk(2, 0));                                 \
            outv = dmul(dmul(poly_eval_d(coef[m_], ncoef[m_], r),                          \
                             poly_eval_d(jac2[jj], njac2[jj], s)), dpowi(hs, m_));         \
        }                                                                                  \
    } while (0)

    for (int i = 0; i < nen; ++i)
        for (int j = 0; j < nen; ++j) {
            dual v;
            BASIS(j, &nodes[3 * i], -1, v);
            V[i * nen + j] = v.f;
        }
    for (int i = 0; i < nen; ++i)
        for (int j = 0; j < nen; ++j) VT[i * nen + j] = V[j * nen + i];
    lu_factor(VT, nen, piv);
    for (int q = 0; q < nq; ++q) {
        double rhs[OR_MAX_NEN], sol[OR_MAX_NEN];
        double grhs[3][OR_MAX_NEN];
        for (int j = 0; j < nen; ++j) {
            dual v;
            BASIS(j, &qpts[3 * q], -1, v);
            rhs[j] = v.f;
            for (int d = 0; d < dim; ++d) {
                BASIS(j, &qpts[3 * q], d, v);
                grhs[d][j] = v.d;
            }
        }
        lu_solve(VT, nen, piv, rhs, sol);
        for (int a = 0; a < nen; ++a) N[q * nen + a] = sol[a];
        for (int d = 0; d < dim; ++d) {
            lu_solve(VT, nen, piv, grhs[d], sol);
            for (int a = 0; a < nen; ++a) dN[(q * nen + a) * dim + d] = sol[a];
        }
    }
    #undef BASIS
    free(V);
    return nen;
}

/* ===================================================================== */
/* DoFManager                                                              */
/* ===================================================================== */

/* CellType -> ElementType (src/utils/DoFManager.cpp:107-140). */
static void cell_to_element(int ct, int *topo, int *tdim) {
    switch (ct) {
    case OR_LINE2: *topo = OR_TENSOR; *tdim = 1; break;
    case OR_TRI3: *topo = OR_SIMPLEX; *tdim = 2; break;
    case OR_TET4: *topo = OR_SIMPLEX; *tdim = 3; break;
    case OR_QUAD4: *topo = OR_TENSOR; *tdim = 2; break;
    case OR_HEX8: *topo = OR_TENSOR; *tdim = 3; break;
    default: *topo = OR_NONE; *tdim = 0; break;
    }
}

/* Map a local point to physical space from the cell's corners
 * (src/utils/DoFManager.cpp:296-338), same operation order. */
static void interpolate_from_corners(const double *xl, const double *c, int ct, double *out) {
    for (int k = 0; k < 3; ++k) {
        double x0 = xl[0], x1 = xl[1], x2 = xl[2];
        switch (ct) {
        case OR_TRI3:
            out[k] = (1 - x0 - x1) * c[0 * 3 + k] + x0 * c[1 * 3 + k] + x1 * c[2 * 3 + k];
            break;
        case OR_TET4:
            out[k] = (1 - x0 - x1 - x2) * c[0 * 3 + k] + x0 * c[1 * 3 + k] + x1 * c[2 * 3 + k] +
                     x2 * c[3 * 3 + k];
            break;
        case OR_QUAD4:
            out[k] = (1.0 / 4.0) * ((1 - x0) * (1 - x1) * c[0 * 3 + k] + (1 + x0) * (1 - x1) * c[1 * 3 + k] +
                                    (1 + x0) * (1 + x1) * c[2 * 3 + k] + (1 - x0) * (1 + x1) * c[3 * 3 + k]);
            break;
        case OR_HEX8:
            out[k] = (1.0 / 8.0) * ((1 - x0) * (1 - x1) * (1 - x2) * c[0 * 3 + k] +
                                    (1 + x0) * (1 - x1) * (1 - x2) * c[1 * 3 + k] +
                                    (1 + x0) * (1 + x1) * (1 - x2) * c[2 * 3 + k] +
                                    (1 - x0) * (1 + x1) * (1 - x2) * c[3 * 3 + k] +
                                    (1 - x0) * (1 - x1) * (1 + x2) * c[4 * 3 + k] +
                                    (1 + x0) * (1 - x1) * (1 + x2) * c[5 * 3 + k] +
                                    (1 + x0) * (1 + x1) * (1 + x2) * c[6 * 3 + k] +
                                    (1 - x0) * (1 + x1) * (1 + x2) * c[7 * 3 + k]);
            break;
        default: out[k] = 0; break;
        }
    }
}

static const double *g_sort_keys; /* snapped coords, 3 per raw node */
static int cmp_snapped_zyx(const void *pa, const void *pb) {
    int a = *(const int *)pa, b = *(const int *)pb;
    const double *ka = g_sort_keys + 3 * (int64_t)a, *kb = g_sort_keys + 3 * (int64_t)b;
    for (int k = 2; k >= 0; --k) {
        if (ka[k] < kb[k]) return -1;
        if (ka[k] > kb[k]) return 1;
    }
    /* Ties merge below; index order only picks the representative, i.e. which
     * coincident raw node gives the merged node its coordinates.  The reference's
     * std::sort is unstable, so its representative is whatever that sort leaves
     * first; the two agree to rounding except where triangles meet
     * quadrilaterals at p >= 3 (their local nodes are snapped differently), and
     * the parity tests assemble those cases on the reference's own numbering. */
    return (a < b) ? -1 : (a > b);
}

/* DoFManager(M, CG, p): p=1 keeps the mesh numbering (DoFManager.cpp:153-160);
 * p>1 creates every cell's local nodes (make_raw_dofs, :176-229), then merges
 * duplicates by sorting snapped coordinates on (z,y,x) and joining neighbours
 * closer than 1e-6 (recombine_all_duplicates, :340-414). */
or_dofmap *or_dofmanager(const double *xyz, int32_t n_nodes, const int32_t *cell_nodes,
                         const int32_t *cell_offsets, const int32_t *cell_types, int32_t n_cells,
                         int32_t p) {
    if (p < 1) return NULL;
    or_dofmap *d = (or_dofmap *)calloc(1, sizeof(or_dofmap));
    d->n_cells = n_cells;
    d->offsets = (int32_t *)calloc(n_cells + 1, sizeof(int32_t));
    d->topology = (int8_t *)malloc(n_cells > 0 ? n_cells : 1);
    d->topo_dim = (int8_t *)malloc(n_cells > 0 ? n_cells : 1);
    d->poly_order = (int8_t *)malloc(n_cells > 0 ? n_cells : 1);
    for (int c = 0; c < n_cells; ++c) {
        int t, td;
        cell_to_element(cell_types[c], &t, &td);
        d->topology[c] = (int8_t)t; d->topo_dim[c] = (int8_t)td; d->poly_order[c] = (int8_t)p;
    }
    if (p == 1) {
        int64_t ne = cell_offsets[n_cells];
        d->elements = (int32_t *)malloc(sizeof(int32_t) * (ne > 0 ? ne : 1));
        memcpy(d->elements, cell_nodes, sizeof(int32_t) * ne);
        memcpy(d->offsets, cell_offsets, sizeof(int32_t) * (n_cells + 1));
        d->n_nodes = n_nodes;
        d->nodes = (double *)malloc(sizeof(double) * 3 * (n_nodes > 0 ? n_nodes : 1));
        memcpy(d->nodes, xyz, sizeof(double) * 3 * n_nodes);
        return d;
    }
    /* make_raw_dofs */
    int64_t total = 0;
    int nloc_cache[3][4] = {{0}};
    for (int c = 0; c < n_cells; ++c) {
        if (d->topology[c] == OR_NONE) continue;
        double tmp[3 * OR_MAX_NEN];
        int t = d->topology[c], td = d->topo_dim[c];
        if (!nloc_cache[t][td]) nloc_cache[t][td] = or_local_nodes(t, td, p, tmp);
        total += nloc_cache[t][td];
    }
    double *raw = (double *)malloc(sizeof(double) * 3 * (total > 0 ? total : 1));
    d->elements = (int32_t *)malloc(sizeof(int32_t) * (total > 0 ? total : 1));
    int64_t next = 0;
    int offset = 0;
    for (int c = 0; c < n_cells; ++c) {
        int t = d->topology[c], td = d->topo_dim[c];
        if (t == OR_NONE) continue;
        double loc[3 * OR_MAX_NEN], corners[3 * 8];
        int nloc = or_local_nodes(t, td, p, loc);
        int nc = cell_offsets[c + 1] - cell_offsets[c];
        for (int i = 0; i < nc && i < 8; ++i)
            for (int k = 0; k < 3; ++k) corners[3 * i + k] = xyz[3 * (int64_t)cell_nodes[cell_offsets[c] + i] + k];
        for (int a = 0; a < nloc; ++a) {
            interpolate_from_corners(&loc[3 * a], corners, cell_types[c], &raw[3 * next]);
            d->elements[next] = (int32_t)next;
            ++next;
        }
        d->offsets[c] = offset;
        offset += nloc;
    }
    d->offsets[n_cells] = offset;
    /* recombine_all_duplicates */
    int64_t N = total;
    double bmin[3], bmax[3];
    for (int k = 0; k < 3; ++k) { bmin[k] = raw[k]; bmax[k] = raw[k]; }
    for (int64_t i = 0; i < N; ++i)
        for (int k = 0; k < 3; ++k) {
            if (raw[3 * i + k] < bmin[k]) bmin[k] = raw[3 * i + k];
            if (raw[3 * i + k] > bmax[k]) bmax[k] = raw[3 * i + k];
        }
    double max_dim = bmax[0] - bmin[0];
    for (int k = 1; k < 3; ++k) if (bmax[k] - bmin[k] > max_dim) max_dim = bmax[k] - bmin[k];
    double snapv = max_dim * 1.0e-6;
    double *keys = (double *)malloc(sizeof(double) * 3 * (N > 0 ? N : 1));
    int *idxs = (int *)malloc(sizeof(int) * (N > 0 ? N : 1));
    for (int64_t i = 0; i < N; ++i) {
        idxs[i] = (int)i;
        /* round(x * (1/s)) * s: the reference's tensor division by a scalar
         * multiplies by the reciprocal (tensor_functions/operators.hpp:66-70) */
        for (int k = 0; k < 3; ++k) keys[3 * i + k] = round(raw[3 * i + k] * (1.0 / snapv)) * snapv;
    }
    g_sort_keys = keys;
    qsort(idxs, N, sizeof(int), cmp_snapped_zyx);
    int *group = (int *)malloc(sizeof(int) * (N > 0 ? N : 1)); /* new number of sorted position i */
    int *first = (int *)malloc(sizeof(int) * (N > 0 ? N : 1));
    int ng = 0;
    for (int64_t i = 0; i < N; ++i) {
        int newg = 1;
        if (i > 0) {
            const double *a = &raw[3 * (int64_t)idxs[i]], *b = &raw[3 * (int64_t)idxs[i - 1]];
            double s = 0;
            for (int k = 0; k < 3; ++k) s += (a[k] - b[k]) * (a[k] - b[k]);
            if (sqrt(s) < 1.0e-6) newg = 0;
        }
        if (newg) first[ng++] = idxs[i];
        group[i] = ng - 1;
    }
    int *raw_to_new = (int *)malloc(sizeof(int) * (N > 0 ? N : 1));
    for (int64_t i = 0; i < N; ++i) raw_to_new[idxs[i]] = group[i];
    d->n_nodes = ng;
    d->nodes = (double *)malloc(sizeof(double) * 3 * (ng > 0 ? ng : 1));
    for (int g = 0; g < ng; ++g)
        for (int k = 0; k < 3; ++k) d->nodes[3 * g + k] = raw[3 * (int64_t)first[g] + k];
    for (int64_t i = 0; i < N; ++i) d->elements[i] = raw_to_new[d->elements[i]];
    free(raw); free(keys); free(idxs); free(group); free(first); free(raw_to_new);
    return d;
}

void or_free_dofmap(or_dofmap *d) {
    if (!d) return;
    free(d->nodes); free(d->offsets); free(d->elements);
    free(d->topology); free(d->topo_dim); free(d->poly_order);
    free(d);
}

/* ===================================================================== */
/* Assembly                                                                */
/* ===================================================================== */

typedef struct {
    int ok, nen, nq, dim;
    double w[OR_MAX_NQ];
    double *N;  /* nq*nen */
    double *dN; /* nq*nen*dim */
} or_eltab;

static void build_eltab(or_eltab *T, int topo, int dim, int p) {
    double qp[3 * OR_MAX_NQ];
    T->nq = or_element_rule(topo, dim, p, qp, T->w);
    double tmp[3 * OR_MAX_NEN];
    T->nen = or_local_nodes(topo, dim, p, tmp);
    T->dim = dim;
    T->N = (double *)malloc(sizeof(double) * T->nq * T->nen);
    T->dN = (double *)malloc(sizeof(double) * T->nq * T->nen * dim);
    or_shape_functions(topo, dim, p, qp, T->nq, T->N, T->dN);
    T->ok = 1;
}

/* Element::update<NSD> (include/element/Element.hpp:109-149) with the closed
 * form det/inverse of include/lin_alg/tensor/tensor_functions/
 * rank2_specializations.hpp:117-177. grad is nen*nsd. */
static double element_update(int nsd, int nen, const double *xe, const double *dNq, int dim,
                             double wq, double *grad) {
    double J[3][3] = {{0}};
    for (int A = 0; A < nen; ++A)
        for (int i = 0; i < nsd; ++i)
            for (int j = 0; j < nsd; ++j) J[i][j] += xe[3 * A + i] * dNq[A * dim + j];
    double det, Ji[3][3];
    if (nsd == 1) {
        det = J[0][0];
        Ji[0][0] = 1.0 / J[0][0];
    } else if (nsd == 2) {
        det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
        double di = 1.0 / det;
        Ji[0][0] = J[1][1] * di; Ji[1][1] = J[0][0] * di;
        Ji[0][1] = -J[0][1] * di; Ji[1][0] = -J[1][0] * di;
    } else {
        det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
              J[0][1] * (J[1][0] * J[2][2] - J[2][0] * J[1][2]) +
              J[0][2] * (J[1][0] * J[2][1] - J[2][0] * J[1][1]);
        double di = 1.0 / det;
        Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) * di;
        Ji[0][1] = -(J[0][1] * J[2][2] - J[2][1] * J[0][2]) * di;
        Ji[0][2] = (J[0][1] * J[1][2] - J[1][1] * J[0][2]) * di;
        Ji[1][0] = -(J[1][0] * J[2][2] - J[2][0] * J[1][2]) * di;
        Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * di;
        Ji[1][2] = -(J[0][0] * J[1][2] - J[1][0] * J[0][2]) * di;
        Ji[2][0] = (J[1][0] * J[2][1] - J[2][0] * J[1][1]) * di;
        Ji[2][1] = -(J[0][0] * J[2][1] - J[2][0] * J[0][1]) * di;
        Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * di;
    }
    for (int A = 0; A < nen; ++A)
        for (int d = 0; d < nsd; ++d) {
            double s = 0;
            for (int j = 0; j < nsd; ++j) s += Ji[j][d] * dNq[A * dim + j];
            grad[A * nsd + d] = s;
        }
    return det * wq;
}

/* Element tangent and residual for one quadrature point. */
static void physics_qp(int physics, int nsd, int nen, int dpn, const double *params,
                       const double *Nq, const double *g, double jxw, double *Ke, double *Re) {
    int nd = nen * dpn;
    if (physics == OR_POISSON) {
        /* apps/BasicPoisson/main.cpp:31-60 (sign is -1 there; +1 gives the SPD
         * form of experimental/sandbox.cpp:17-35) */
        double sign = params[0], f = params[1];
        for (int A = 0; A < nen; ++A)
            for (int B = A; B < nen; ++B) {
                double dt = 0;
                for (int d = 0; d < nsd; ++d) dt += g[A * nsd + d] * g[B * nsd + d];
                Ke[A * nd + B] += sign * (dt * jxw);
                Ke[B * nd + A] = Ke[A * nd + B];
            }
        if (Re) for (int A = 0; A < nen; ++A) Re[A] += (f * jxw) * Nq[A];
    } else if (physics == OR_ELASTICITY) {
        /* apps/BasicLinearElasticity/main.cpp:53-112:
         * K_{Ai,Bk} -= C_{ikjl} dN_A/dx_j dN_B/dx_l jxw with
         * C_{ikjl} = lambda d_ij d_kl + mu (d_ik d_jl + d_il d_jk) */
        double sign = params[0], lam = params[1], mu = params[2];
        for (int An = 0; An < nen; ++An) {
            const double *gA = &g[An * nsd];
            for (int i = 0; i < nsd; ++i) {
                int A = An * nsd + i;
                for (int Bn = An; Bn < nen; ++Bn) {
                    const double *gB = &g[Bn * nsd];
                    for (int k = 0; k < nsd; ++k) {
                        int B = Bn * nsd + k;
                        double dt = 0;
                        for (int j = 0; j < nsd; ++j)
                            for (int l = 0; l < nsd; ++l) {
                                double C = lam * (i == j) * (k == l) + mu * ((i == k) * (j == l) + (i == l) * (j == k));
                                dt += C * (gA[j] * gB[l]);
                            }
                        Ke[A * nd + B] += sign * (dt * jxw);
                        if (Bn != An) Ke[B * nd + A] = Ke[A * nd + B];
                    }
                }
            }
        }
        if (Re)
            for (int A = 0; A < nen * nsd; ++A) Re[A] += params[3 + (A % nsd)] * Nq[A / nsd] * jxw;
    } else if (physics == OR_SUPG) {
        /* apps/supg_learning/supg_advection.hpp:25-122 (steady): Galerkin
         * advection with U=(U0,0,0) plus streamline-diffusion tensor
         * k I + alpha h/(2|U|) U (x) U, alpha = coth(Pe) - 1/Pe, Pe = U0 h/(2k).
         * The advection term is summed inside the Acomp loop, as the reference does. */
        double kdiff = params[0], h = params[1], U0 = params[2], Q = params[3];
        double Pe = U0 * h / (2 * kdiff);
        double alpha = (Pe == 0) ? 0.0 : cosh(Pe) / sinh(Pe) - 1.0 / Pe;
        double U[3] = {U0, 0, 0};
        double normU = 0;
        for (int d = 0; d < nsd; ++d) normU += U[d] * U[d];
        normU = sqrt(normU);
        double Kd[3][3];
        for (int a = 0; a < nsd; ++a)
            for (int b = 0; b < nsd; ++b) Kd[a][b] = (a == b) ? kdiff : 0.0;
        if (normU > 0)
            for (int a = 0; a < nsd; ++a)
                for (int b = 0; b < nsd; ++b) Kd[a][b] += (alpha * h / (normU * 2)) * (U[a] * U[b]);
        for (int A = 0; A < nen; ++A)
            for (int Ac = 0; Ac < nsd; ++Ac)
                for (int B = 0; B < nen; ++B)
                    for (int Bc = 0; Bc < nsd; ++Bc)
                        Ke[A * nd + B] += (Nq[A] * U[Bc] * g[B * nsd + Bc] +
                                           g[A * nsd + Ac] * g[B * nsd + Bc] * Kd[Ac][Bc]) * jxw;
        if (Re) {
            double Uhat[3] = {0, 0, 0};
            if (normU > 0)
                for (int d = 0; d < nsd; ++d) Uhat[d] = (alpha * h / 2) * U[d] / normU;
            for (int A = 0; A < nen; ++A)
                for (int Ac = 0; Ac < nsd; ++Ac) Re[A] -= (Nq[A] * Q + Uhat[Ac] * g[A * nsd + Ac]) * jxw;
        }
    }
}

typedef struct { int64_t col; double val; int64_t ord; } or_entry;
static int cmp_entry(const void *a, const void *b) {
    const or_entry *x = (const or_entry *)a, *y = (const or_entry *)b;
    if (x->col != y->col) return x->col < y->col ? -1 : 1;
    return (x->ord < y->ord) ? -1 : (x->ord > y->ord);
}

/* Sort each row's (col,val) list by column, keeping emission order among
 * duplicates, and sum duplicates in that order.  bucket sizes in cnt. */
static or_csr *compress_rows(int64_t nrows, int64_t ncols, const int64_t *start, or_entry *ent) {
    or_csr *A = (or_csr *)calloc(1, sizeof(or_csr));
    A->nrows = nrows; A->ncols = ncols;
    A->row_ptr = (int64_t *)calloc(nrows + 1, sizeof(int64_t));
    int64_t *uniq = (int64_t *)calloc(nrows > 0 ? nrows : 1, sizeof(int64_t));
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t r = 0; r < nrows; ++r) {
        int64_t b = start[r], e = start[r + 1];
        for (int64_t i = b; i < e; ++i) ent[i].ord = i;
        qsort(ent + b, e - b, sizeof(or_entry), cmp_entry);
        int64_t u = 0;
        for (int64_t i = b; i < e; ++i) {
            if (i == b || ent[i].col != ent[b + u - 1].col) { ent[b + u] = ent[i]; ++u; }
            else ent[b + u - 1].val += ent[i].val;
        }
        uniq[r] = u;
    }
    for (int64_t r = 0; r < nrows; ++r) A->row_ptr[r + 1] = A->row_ptr[r] + uniq[r];
    A->nnz = A->row_ptr[nrows];
    A->col = (int64_t *)malloc(sizeof(int64_t) * (A->nnz > 0 ? A->nnz : 1));
    A->val = (double *)malloc(sizeof(double) * (A->nnz > 0 ? A->nnz : 1));
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t r = 0; r < nrows; ++r)
        for (int64_t i = 0; i < uniq[r]; ++i) {
            A->col[A->row_ptr[r] + i] = ent[start[r] + i].col;
            A->val[A->row_ptr[r] + i] = ent[start[r] + i].val;
        }
    free(uniq);
    return A;
}

/* CGAssembly<Physics> (include/assembly/CGAssembly.hpp:27-186): element loop,
 * quadrature loop with Element::update, physics callbacks, emission of every
 * (nen*dpn)^2 entry, duplicate summation in element order. */
or_csr *or_assemble(const or_dofmap *d, int32_t dpn, int32_t nsd, int32_t physics,
                    const double *params, double *residual) {
    or_eltab tabs[3][4];
    memset(tabs, 0, sizeof(tabs));
    int64_t ndofs = (int64_t)d->n_nodes * dpn;
    int32_t nc = d->n_cells;
    /* per-node incident (element, nen) in ascending element order */
    int64_t *nstart = (int64_t *)calloc(d->n_nodes + 1, sizeof(int64_t));
    for (int e = 0; e < nc; ++e) {
        if (d->topo_dim[e] != nsd || d->topology[e] == OR_NONE) continue;
        for (int i = d->offsets[e]; i < d->offsets[e + 1]; ++i) nstart[d->elements[i] + 1]++;
    }
    for (int n = 0; n < d->n_nodes; ++n) nstart[n + 1] += nstart[n];
    int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (d->n_nodes + 1));
    memcpy(fill, nstart, sizeof(int64_t) * (d->n_nodes + 1));
    int32_t *adj = (int32_t *)malloc(sizeof(int32_t) * (nstart[d->n_nodes] > 0 ? nstart[d->n_nodes] : 1));
    for (int e = 0; e < nc; ++e) {
        if (d->topo_dim[e] != nsd || d->topology[e] == OR_NONE) continue;
        for (int i = d->offsets[e]; i < d->offsets[e + 1]; ++i) adj[fill[d->elements[i]]++] = e;
    }
    /* row bucket sizes: every incident element contributes nen*dpn entries to each
     * of the node's dpn rows; an element listing a node twice contributes twice. */
    int64_t *rstart = (int64_t *)calloc(ndofs + 1, sizeof(int64_t));
    for (int n = 0; n < d->n_nodes; ++n) {
        int64_t s = 0;
        for (int64_t j = nstart[n]; j < nstart[n + 1]; ++j) {
            int e = adj[j];
            s += (int64_t)(d->offsets[e + 1] - d->offsets[e]) * dpn;
        }
        for (int c = 0; c < dpn; ++c) rstart[(int64_t)n * dpn + c + 1] = s;
    }
    for (int64_t r = 0; r < ndofs; ++r) rstart[r + 1] += rstart[r];
    or_entry *ent = (or_entry *)malloc(sizeof(or_entry) * (rstart[ndofs] > 0 ? rstart[ndofs] : 1));
    /* element order position of each (node, element incidence) */
    for (int e = 0; e < nc; ++e) {
        if (d->topo_dim[e] != nsd || d->topology[e] == OR_NONE) continue;
        int t = d->topology[e], td = d->topo_dim[e];
        if (!tabs[t][td].ok) build_eltab(&tabs[t][td], t, td, d->poly_order[e]);
    }
    if (residual) memset(residual, 0, sizeof(double) * ndofs);
    /* The write position of element e in node n's bucket is the sum of the sizes
     * of the incident elements before it.  Compute per incidence. */
    int64_t *incpos = (int64_t *)malloc(sizeof(int64_t) * (nstart[d->n_nodes] > 0 ? nstart[d->n_nodes] : 1));
    for (int n = 0; n < d->n_nodes; ++n) {
        int64_t s = 0;
        for (int64_t j = nstart[n]; j < nstart[n + 1]; ++j) {
            incpos[j] = s;
            int e = adj[j];
            s += (int64_t)(d->offsets[e + 1] - d->offsets[e]) * dpn;
        }
    }
    double *Rall = residual ? (double *)calloc((size_t)(d->offsets[nc] > 0 ? d->offsets[nc] : 1) * dpn, sizeof(double)) : NULL;
#pragma omp parallel for schedule(dynamic, 16)
    for (int e = 0; e < nc; ++e) {
        if (d->topo_dim[e] != nsd || d->topology[e] == OR_NONE) continue;
        const or_eltab *T = &tabs[d->topology[e]][d->topo_dim[e]];
        int nen = d->offsets[e + 1] - d->offsets[e];
        const int32_t *gn = &d->elements[d->offsets[e]];
        int nd = nen * dpn;
        double *Ke = (double *)calloc((size_t)nd * nd, sizeof(double));
        double Re[OR_MAX_NEN * 3];
        memset(Re, 0, sizeof(Re));
        double xe[3 * OR_MAX_NEN], grad[3 * OR_MAX_NEN];
        for (int A = 0; A < nen; ++A)
            for (int k = 0; k < 3; ++k) xe[3 * A + k] = d->nodes[3 * (int64_t)gn[A] + k];
        for (int q = 0; q < T->nq; ++q) {
            double jxw = element_update(nsd, nen, xe, &T->dN[(int64_t)q * nen * T->dim], T->dim, T->w[q], grad);
            physics_qp(physics, nsd, nen, dpn, params, &T->N[(int64_t)q * nen], grad, jxw, Ke, Re);
        }
        /* scatter: entry (A,B) goes to row GA's bucket at the element's slot */
        for (int a = 0; a < nen; ++a) {
            int node = gn[a];
            /* find this incidence's position (first unused match for repeated nodes) */
            int64_t pos = -1;
            for (int64_t j = nstart[node]; j < nstart[node + 1]; ++j)
                if (adj[j] == e) { pos = incpos[j]; break; }
            for (int ca = 0; ca < dpn; ++ca) {
                int A = a * dpn + ca;
                int64_t GA = (int64_t)node * dpn + ca;
                or_entry *dst = ent + rstart[GA] + pos;
                for (int B = 0; B < nd; ++B) {
                    dst[B].col = (int64_t)gn[B / dpn] * dpn + (B % dpn);
                    dst[B].val = Ke[A * nd + B];
                }
            }
        }
        if (Rall)
            for (int A = 0; A < nd; ++A) Rall[(int64_t)d->offsets[e] * dpn + A] = Re[A];
        free(Ke);
    }
    if (residual) {
        for (int e = 0; e < nc; ++e) {
            if (d->topo_dim[e] != nsd || d->topology[e] == OR_NONE) continue;
            int nen = d->offsets[e + 1] - d->offsets[e];
            for (int A = 0; A < nen * dpn; ++A)
                residual[(int64_t)d->elements[d->offsets[e] + A / dpn] * dpn + A % dpn] +=
                    Rall[(int64_t)d->offsets[e] * dpn + A];
        }
        free(Rall);
    }
    or_csr *K = compress_rows(ndofs, ndofs, rstart, ent);
    free(ent); free(rstart); free(incpos); free(adj); free(fill); free(nstart);
    for (int t = 0; t < 3; ++t)
        for (int td = 0; td < 4; ++td)
            if (tabs[t][td].ok) { free(tabs[t][td].N); free(tabs[t][td].dN); }
    return K;
}

/* LocalSmoothingGradient<Physics> (include/assembly/LocalSmoothingGradient.hpp:20-94):
 * over the cells of topology dimension nsd in cell order and their quadrature
 * points in order, the gradient of each solution component at the point
 * (qp_grad(comp, i) = sum over local dofs A of u_A dN_A/dx_i) is spread to the
 * element's dofs with weights N_A jxw into VolTimesGrad, and N_A jxw into Volume;
 * the result is VolTimesGrad / Volume per dof (0/0 where no cell touches it). */
void or_local_smoothing_gradient(const or_dofmap *d, int32_t dpn, int32_t nsd, const double *sol, double *grad) {
    or_eltab tabs[3][4];
    memset(tabs, 0, sizeof(tabs));
    const int64_t ndofs = (int64_t)d->n_nodes * dpn;
    double *vol = (double *)calloc(ndofs > 0 ? ndofs : 1, sizeof(double));
    double *vtg = (double *)calloc(ndofs > 0 ? ndofs * nsd : 1, sizeof(double));
    for (int e = 0; e < d->n_cells; ++e) {
        if (d->topo_dim[e] != nsd || d->topology[e] == OR_NONE) continue;
        or_eltab *T = &tabs[d->topology[e]][d->topo_dim[e]];
        if (!T->ok) build_eltab(T, d->topology[e], d->topo_dim[e], d->poly_order[e]);
        const int nen = d->offsets[e + 1] - d->offsets[e];
        const int32_t *gn = &d->elements[d->offsets[e]];
        double xe[3 * OR_MAX_NEN], g[3 * OR_MAX_NEN], ul[3 * OR_MAX_NEN];
        for (int A = 0; A < nen; ++A)
            for (int k = 0; k < 3; ++k) xe[3 * A + k] = d->nodes[3 * (int64_t)gn[A] + k];
        for (int A = 0; A < nen * dpn; ++A) ul[A] = sol[(int64_t)gn[A / dpn] * dpn + A % dpn];
        for (int q = 0; q < T->nq; ++q) {
            const double jxw = element_update(nsd, nen, xe, &T->dN[(int64_t)q * nen * T->dim], T->dim, T->w[q], g);
            double qg[3][3] = {{0}};
            for (int A = 0; A < nen * dpn; ++A)
                for (int i = 0; i < nsd; ++i) qg[A % dpn][i] += ul[A] * g[(A / dpn) * nsd + i];
            const double *Nq = &T->N[(int64_t)q * nen];
            for (int A = 0; A < nen * dpn; ++A) {
                const int64_t G = (int64_t)gn[A / dpn] * dpn + A % dpn;
                const double NA = Nq[A / dpn];
                vol[G] += NA * jxw;
                for (int i = 0; i < nsd; ++i) vtg[G * nsd + i] += NA * qg[A % dpn][i] * jxw;
            }
        }
    }
    for (int64_t A = 0; A < ndofs; ++A)
        for (int i = 0; i < nsd; ++i) grad[A * nsd + i] = vtg[A * nsd + i] / vol[A];
    free(vol);
    free(vtg);
    for (int t = 0; t < 3; ++t)
        for (int td = 0; td < 4; ++td)
            if (tabs[t][td].ok) { free(tabs[t][td].N); free(tabs[t][td].dN); }
}

/* DirichletBC::apply, RowMajor form (src/boundary_conditions/DirichletBC.cpp:27-56):
 * rhs -= A g, then zero BC rows and columns, unit diagonal, rhs_bc = g. */
void or_dirichlet_apply(or_csr *A, double *rhs, const uint8_t *mask, const double *vals) {
    int64_t n = A->nrows;
    double *g = (double *)calloc(n, sizeof(double));
    for (int64_t i = 0; i < n; ++i) if (mask[i]) g[i] = vals[i];
    double *Ag = (double *)malloc(sizeof(double) * n);
    or_csr_spmv(A, g, Ag);
    for (int64_t i = 0; i < n; ++i) rhs[i] -= Ag[i];
    for (int64_t r = 0; r < n; ++r)
        for (int64_t k = A->row_ptr[r]; k < A->row_ptr[r + 1]; ++k) {
            int64_t c = A->col[k];
            if (mask[r] || mask[c]) {
                A->val[k] = 0;
                if (r == c) { rhs[r] = g[c]; A->val[k] = 1; }
            }
        }
    free(g); free(Ag);
}

/* ===================================================================== */
/* Sparse containers                                                       */
/* ===================================================================== */

typedef struct { int64_t r, c; double v; } trip;
static int cmp_trip_rcv(const void *a, const void *b) {
    const trip *x = (const trip *)a, *y = (const trip *)b;
    if (x->r != y->r) return x->r < y->r ? -1 : 1;
    if (x->c != y->c) return x->c < y->c ? -1 : 1;
    if (x->v != y->v) return x->v < y->v ? -1 : 1;
    return 0;
}

/* sparse_csr(triplets): sort by (row, col, value), sum duplicates in that order
 * (include/old_handmade_linalg/sparse_csr.hpp:90-149). Rows and columns are the
 * maxima + 1. */
or_csr *or_csr_from_triplets(const int64_t *r, const int64_t *c, const double *v, int64_t n) {
    or_csr *A = (or_csr *)calloc(1, sizeof(or_csr));
    if (n == 0) {
        A->row_ptr = (int64_t *)calloc(1, sizeof(int64_t));
        A->col = (int64_t *)malloc(sizeof(int64_t)); A->val = (double *)malloc(sizeof(double));
        return A;
    }
    trip *t = (trip *)malloc(sizeof(trip) * n);
    int64_t mr = 0, mc = 0;
    for (int64_t i = 0; i < n; ++i) {
        t[i].r = r[i]; t[i].c = c[i]; t[i].v = v[i];
        if (r[i] > mr) mr = r[i];
        if (c[i] > mc) mc = c[i];
    }
    qsort(t, n, sizeof(trip), cmp_trip_rcv);
    A->nrows = mr + 1; A->ncols = mc + 1;
    A->row_ptr = (int64_t *)calloc(A->nrows + 1, sizeof(int64_t));
    A->col = (int64_t *)malloc(sizeof(int64_t) * n);
    A->val = (double *)malloc(sizeof(double) * n);
    int64_t k = -1;
    for (int64_t i = 0; i < n; ++i) {
        if (k >= 0 && t[i].r == t[i - 1].r && t[i].c == t[i - 1].c) { A->val[k] += t[i].v; continue; }
        ++k;
        A->col[k] = t[i].c; A->val[k] = t[i].v;
        A->row_ptr[t[i].r + 1]++;
    }
    A->nnz = k + 1;
    for (int64_t i = 0; i < A->nrows; ++i) A->row_ptr[i + 1] += A->row_ptr[i];
    free(t);
    return A;
}

static int g_block;
static int cmp_trip_bcsr(const void *a, const void *b) {
    const trip *x = (const trip *)a, *y = (const trip *)b;
    int64_t B = g_block;
    int64_t k1[4] = {x->r / B, x->c / B, x->r % B, x->c % B};
    int64_t k2[4] = {y->r / B, y->c / B, y->r % B, y->c % B};
    for (int i = 0; i < 4; ++i) if (k1[i] != k2[i]) return k1[i] < k2[i] ? -1 : 1;
    return 0;
}

/* sparse_bcsr<BLOCK>(triplets): sort by (I,J,i,j), one block per distinct
 * (I,J), values row-major inside a block, duplicates summed
 * (include/old_handmade_linalg/sparse_bcsr.hpp:93-176). */
or_bcsr *or_bcsr_from_triplets(int32_t block, const int64_t *r, const int64_t *c,
                               const double *v, int64_t n) {
    or_bcsr *A = (or_bcsr *)calloc(1, sizeof(or_bcsr));
    A->block = block;
    if (n == 0) { A->brow_ptr = (int64_t *)calloc(1, sizeof(int64_t)); return A; }
    trip *t = (trip *)malloc(sizeof(trip) * n);
    int64_t mr = 0, mc = 0;
    for (int64_t i = 0; i < n; ++i) {
        t[i].r = r[i]; t[i].c = c[i]; t[i].v = v[i];
        if (r[i] > mr) mr = r[i];
        if (c[i] > mc) mc = c[i];
    }
    g_block = block;
    qsort(t, n, sizeof(trip), cmp_trip_bcsr);
    int64_t B = block, B2 = B * B;
    A->nbrows = mr / B + 1; A->nbcols = mc / B + 1;
    int64_t nb = 1;
    for (int64_t i = 1; i < n; ++i)
        if (t[i].r / B != t[i - 1].r / B || t[i].c / B != t[i - 1].c / B) ++nb;
    A->nnzb = nb;
    A->brow_ptr = (int64_t *)calloc(A->nbrows + 1, sizeof(int64_t));
    A->bcol = (int64_t *)malloc(sizeof(int64_t) * nb);
    A->val = (double *)calloc(nb * B2, sizeof(double));
    int64_t k = -1;
    for (int64_t i = 0; i < n; ++i) {
        if (i == 0 || t[i].r / B != t[i - 1].r / B || t[i].c / B != t[i - 1].c / B) {
            ++k;
            A->bcol[k] = t[i].c / B;
            A->brow_ptr[t[i].r / B + 1]++;
        }
        A->val[k * B2 + (t[i].r % B) * B + (t[i].c % B)] += t[i].v;
    }
    for (int64_t i = 0; i < A->nbrows; ++i) A->brow_ptr[i + 1] += A->brow_ptr[i];
    free(t);
    return A;
}

/* Block view of a CSR matrix whose pattern is closed under blocks (every
 * block that holds one entry holds all B*B); used to compare block kernels. */
or_bcsr *or_bcsr_from_csr(const or_csr *A, int32_t block) {
    int64_t n = A->nnz;
    int64_t *r = (int64_t *)malloc(sizeof(int64_t) * (n > 0 ? n : 1));
    for (int64_t i = 0; i < A->nrows; ++i)
        for (int64_t k = A->row_ptr[i]; k < A->row_ptr[i + 1]; ++k) r[k] = i;
    or_bcsr *Bm = or_bcsr_from_triplets(block, r, A->col, A->val, n);
    free(r);
    return Bm;
}

void or_free_csr(or_csr *A) { if (A) { free(A->row_ptr); free(A->col); free(A->val); free(A); } }
void or_free_bcsr(or_bcsr *A) { if (A) { free(A->brow_ptr); free(A->bcol); free(A->val); free(A); } }

/* ===================================================================== */
/* SpMV, preconditioners, Krylov solvers                                   */
/* ===================================================================== */

/* csr_spmv: one accumulator per row (include/old_handmade_linalg/csr_spmv.hpp:25-56). */
void or_csr_spmv(const or_csr *A, const double *x, double *y) {
#pragma omp parallel for schedule(static, 128)
    for (int64_t r = 0; r < A->nrows; ++r) {
        double acc = 0;
        for (int64_t k = A->row_ptr[r]; k < A->row_ptr[r + 1]; ++k) acc += A->val[k] * x[A->col[k]];
        y[r] = acc;
    }
}

/* bcsr_spmv: per block row, B accumulators, row-major block walk
 * (include/old_handmade_linalg/bcsr_spmv.hpp:23-62). */
void or_bcsr_spmv(const or_bcsr *A, const double *x, double *y) {
    int64_t B = A->block, B2 = B * B;
#pragma omp parallel for schedule(static, 64)
    for (int64_t br = 0; br < A->nbrows; ++br) {
        double acc[8] = {0};
        for (int64_t k = A->brow_ptr[br]; k < A->brow_ptr[br + 1]; ++k)
            for (int64_t i = 0; i < B; ++i)
                for (int64_t j = 0; j < B; ++j) acc[i] += A->val[k * B2 + i * B + j] * x[A->bcol[k] * B + j];
        for (int64_t i = 0; i < B; ++i) y[br * B + i] = acc[i];
    }
}

/* VectorExpression::dot with four partial sums
 * (include/old_handmade_linalg/VectorExpression.hpp:33-54). */
static double vdot(const double *a, const double *b, int64_t n) {
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    int64_t NN = (n / 4) * 4;
    for (int64_t i = 0; i < NN; i += 4) {
        s0 += a[i] * b[i]; s1 += a[i + 1] * b[i + 1]; s2 += a[i + 2] * b[i + 2]; s3 += a[i + 3] * b[i + 3];
    }
    for (int64_t i = NN; i < n; ++i) s0 += a[i] * b[i];
    return s0 + s1 + s2 + s3;
}

/* ILU(0) without pivoting on the pattern of A; a zero pivot skips that pivot's
 * elimination.  Row-wise (IKJ) ordering of the reference's pivot-major (KIJ)
 * elimination (solver/iterative/ILUPreconditioner.hpp:96-185,256-329); both
 * apply, to each entry, the same updates in the same order. */
or_csr *or_ilu0(const or_csr *A) {
    or_csr *F = (or_csr *)calloc(1, sizeof(or_csr));
    *F = *A;
    F->row_ptr = (int64_t *)malloc(sizeof(int64_t) * (A->nrows + 1));
    F->col = (int64_t *)malloc(sizeof(int64_t) * (A->nnz > 0 ? A->nnz : 1));
    F->val = (double *)malloc(sizeof(double) * (A->nnz > 0 ? A->nnz : 1));
    memcpy(F->row_ptr, A->row_ptr, sizeof(int64_t) * (A->nrows + 1));
    memcpy(F->col, A->col, sizeof(int64_t) * A->nnz);
    memcpy(F->val, A->val, sizeof(double) * A->nnz);
    int64_t n = F->nrows;
    int64_t *diag = (int64_t *)malloc(sizeof(int64_t) * (n > 0 ? n : 1));
    for (int64_t r = 0; r < n; ++r) {
        diag[r] = -1;
        for (int64_t k = F->row_ptr[r]; k < F->row_ptr[r + 1]; ++k)
            if (F->col[k] == r) { diag[r] = k; break; }
    }
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t kk = F->row_ptr[i]; kk < F->row_ptr[i + 1]; ++kk) {
            int64_t k = F->col[kk];
            if (k >= i) break;
            if (k == n - 1) continue;             /* the reference's pivot loop stops at n-2 */
            double piv = diag[k] >= 0 ? F->val[diag[k]] : 0.0;
            if (piv == 0) continue;
            double m = F->val[kk] / piv;
            /* merge row i (cols > k) with row k (cols > k) */
            int64_t pi = kk + 1, pk = diag[k] + 1;
            int64_t ei = F->row_ptr[i + 1], ek = F->row_ptr[k + 1];
            while (pi < ei && pk < ek) {
                if (F->col[pi] == F->col[pk]) { F->val[pi] -= m * F->val[pk]; ++pi; ++pk; }
                else if (F->col[pi] < F->col[pk]) ++pi;
                else ++pk;
            }
            F->val[kk] = m;
        }
    }
    free(diag);
    return F;
}

/* f_subst then b_subst (ILUPreconditioner.hpp:190-253). */
void or_ilu_solve(const or_csr *F, double *z) {
    int64_t n = F->nrows;
    for (int64_t r = 0; r < n; ++r)
        for (int64_t k = F->row_ptr[r]; k < F->row_ptr[r + 1]; ++k) {
            if (F->col[k] >= r) break;
            z[r] -= F->val[k] * z[F->col[k]];
        }
    for (int64_t r = n - 1; r >= 0; --r) {
        int64_t id = 0;
        for (int64_t k = F->row_ptr[r]; k < F->row_ptr[r + 1]; ++k)
            if (F->col[k] == r) { id = k; break; }
        for (int64_t k = id + 1; k < F->row_ptr[r + 1]; ++k) z[r] -= F->val[k] * z[F->col[k]];
        z[r] /= F->val[id];
    }
}

double or_true_relres(const or_csr *A, const double *b, const double *x) {
    int64_t n = A->nrows;
    double *t = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
    or_csr_spmv(A, x, t);
    double rr = 0, bb = 0;
    for (int64_t i = 0; i < n; ++i) { double d = b[i] - t[i]; rr += d * d; bb += b[i] * b[i]; }
    free(t);
    return bb > 0 ? sqrt(rr / bb) : sqrt(rr);
}

/* cg_solve / pcg_solve (solver/iterative/cg_solve.hpp:33-81,
 * pcg_solve.hpp:126-178).  criterion REFERENCE: stop when r^T z / r0^T z0 < tol
 * (z = r without a preconditioner), at most maxiter (default N) iterations.
 * criterion RELRES: stop when ||r|| <= tol ||b||. */
int64_t or_cg(const or_csr *A, const double *b, double *x, int32_t precond, int32_t criterion,
              double tol, int64_t maxiter, double *relres) {
    int64_t n = A->nrows;
    if (maxiter <= 0) maxiter = n;
    double *r = (double *)malloc(sizeof(double) * n), *z = (double *)malloc(sizeof(double) * n);
    double *p = (double *)malloc(sizeof(double) * n), *Ap = (double *)malloc(sizeof(double) * n);
    double *dinv = NULL;
    or_csr *F = NULL;
    if (precond == OR_PRECOND_JACOBI) {
        dinv = (double *)malloc(sizeof(double) * n);
        for (int64_t i = 0; i < n; ++i) {
            double a = 0;
            for (int64_t k = A->row_ptr[i]; k < A->row_ptr[i + 1]; ++k) if (A->col[k] == i) { a = A->val[k]; break; }
            dinv[i] = 1.0 / a;
        }
    } else if (precond == OR_PRECOND_ILU0) {
        F = or_ilu0(A);
    }
    or_csr_spmv(A, x, Ap);
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - Ap[i];
#define APPLY_M(dst, src)                                                       \
    do {                                                                         \
        for (int64_t i = 0; i < n; ++i) dst[i] = src[i];                         \
        if (dinv) for (int64_t i = 0; i < n; ++i) dst[i] *= dinv[i];             \
        if (F) or_ilu_solve(F, dst);                                             \
    } while (0)
    APPLY_M(z, r);
    memcpy(p, z, sizeof(double) * n);
    double rz = vdot(r, z, n), rz0 = rz;
    double bb = vdot(b, b, n);
    int64_t k = 0;
    if (rz != 0) {
        while (k++ < maxiter) {
            or_csr_spmv(A, p, Ap);
            double alpha = rz / vdot(p, Ap, n);
            for (int64_t i = 0; i < n; ++i) x[i] += p[i] * alpha;
            for (int64_t i = 0; i < n; ++i) r[i] += -alpha * Ap[i];
            APPLY_M(z, r);
            double rzn = vdot(r, z, n);
            if (criterion == OR_CRIT_REFERENCE) {
                if (rzn / rz0 < tol) break;
            } else {
                double rr = vdot(r, r, n);
                if (sqrt(rr) <= tol * sqrt(bb)) break;
            }
            double beta = rzn / rz;
            rz = rzn;
            for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        }
    } else {
        k = 0;
    }
#undef APPLY_M
    if (relres) *relres = or_true_relres(A, b, x);
    free(r); free(z); free(p); free(Ap); free(dinv);
    if (F) or_free_csr(F);
    return k > maxiter ? maxiter : k;
}

/* bicgstab_solve (solver/iterative/bicgstab_solve.hpp:215-283), unpreconditioned.
 * criterion REFERENCE: true residual ||Ax-b||^2/||b||^2 < tol checked every
 * max(N/100,1) iterations; if b.b < tol the reference returns b itself.
 * criterion RELRES: recursive residual checked every iteration. maxiter caps
 * the loop (the reference has no cap). */
int64_t or_bicgstab(const or_csr *A, const double *b, double *x, int32_t criterion, double tol,
                    int64_t maxiter, double *relres) {
    int64_t n = A->nrows;
    if (maxiter <= 0) maxiter = 100 * n + 1000;
    double *r = (double *)malloc(sizeof(double) * n), *rhat = (double *)malloc(sizeof(double) * n);
    double *v = (double *)calloc(n, sizeof(double)), *p = (double *)calloc(n, sizeof(double));
    double *s = (double *)malloc(sizeof(double) * n), *t = (double *)malloc(sizeof(double) * n);
    double *tmp = (double *)malloc(sizeof(double) * n);
    or_csr_spmv(A, x, tmp);
    for (int64_t i = 0; i < n; ++i) { r[i] = b[i] - tmp[i]; rhat[i] = r[i]; }
    int64_t freq = (n / 100 > 1) ? n / 100 : 1;
    double res0 = vdot(b, b, n);
    int64_t k = 0, its = 0;
    if (criterion == OR_CRIT_REFERENCE && res0 < tol) {
        memcpy(x, b, sizeof(double) * n);
    } else {
        double rho_old = 1, alpha = 1, w_old = 1;
        while (its < maxiter) {
            ++its;
            double rho_new = vdot(rhat, r, n);
            double beta = (rho_new / rho_old) * (alpha / w_old);
            for (int64_t i = 0; i < n; ++i) p[i] = r[i] + p[i] * beta - v[i] * (w_old * beta);
            or_csr_spmv(A, p, v);
            alpha = rho_new / vdot(rhat, v, n);
            for (int64_t i = 0; i < n; ++i) s[i] = r[i] - v[i] * alpha;
            or_csr_spmv(A, s, t);
            double tt = vdot(t, t, n);
            double w_new = (tt == 0) ? 0 : vdot(t, s, n) / tt;
            for (int64_t i = 0; i < n; ++i) x[i] += p[i] * alpha + s[i] * w_new;
            if (criterion == OR_CRIT_REFERENCE) {
                if (k % freq == 0) {
                    or_csr_spmv(A, x, tmp);
                    double res = 0;
                    for (int64_t i = 0; i < n; ++i) { double d = tmp[i] - b[i]; res += d * d; }
                    if (res / res0 < tol) break;
                }
            }
            for (int64_t i = 0; i < n; ++i) r[i] = s[i] - t[i] * w_new;
            if (criterion == OR_CRIT_RELRES) {
                double rr = vdot(r, r, n);
                if (sqrt(rr) <= tol * sqrt(res0)) break;
            }
            rho_old = rho_new;
            w_old = w_new;
            ++k;
        }
    }
    if (relres) *relres = or_true_relres(A, b, x);
    free(r); free(rhat); free(v); free(p); free(s); free(t); free(tmp);
    return its;
}
