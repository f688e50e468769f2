// host_fe.cpp -- quadrature, reference elements, CG DoF numbering and element
// colouring on the host.
#include "host_fe.h"

#ifdef _OPENMP
#include <omp.h>
#endif

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>

namespace yg {

// Gauss-Legendre points: Newton on P_n from -cos(pi (i+0.75)/(n+0.5)) until
// |P_n| <= 1e-15 (the reference's iteration, src/quadrature/QuadratureRule.cpp:66-106,
// kept step for step so the points are bit-identical).
void gauss_legendre_1d(int n, double *x, double *w) {
    const double PI = std::atan2(1., 1.) * 4;
    for (int i = 0; i < n; ++i) {
        double xx = -std::cos(PI * (1 + i - 0.25) / (n + 0.5));
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
        } while (std::fabs(Pn) > 1.0e-15 && ++guard < 200);
        x[i] = xx;
        w[i] = 2.0 / ((1 - xx * xx) * (dP * dP));
    }
}

// Gauss-Lobatto points by the reference's fixed-point iteration
// (src/quadrature/QuadratureRule.cpp:25-63).
void gauss_lobatto_1d(int n, double *x, double *w) {
    const double PI = std::atan2(1., 1.) * 4;
    for (int i = 0; i < n; ++i) {
        double xx = -std::cos((PI * i) / (n - 1));
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
        } while (std::fabs(xx - xold) > 1.0e-15 && ++guard < 200);
        x[i] = xx;
        w[i] = 2 / (n * (n - 1) * Pn * Pn);
    }
}

// QuadratureRule::make_tensor_product (src/quadrature/QuadratureRule.cpp:109-175):
// points per direction chosen for exactness `order`, x fastest.
int tensor_rule(bool lobatto, int dim, int order, std::vector<double> &pts, std::vector<double> &w) {
    pts.clear();
    w.clear();
    if (dim == 0) {
        pts = {0, 0, 0};
        w = {1};
        return 1;
    }
    double x1[64], w1[64];
    int n;
    if (!lobatto) {
        n = (order + 1) / 2 + (order + 1) % 2;
        gauss_legendre_1d(n, x1, w1);
    } else {
        n = (order + 3) / 2 + (order + 3) % 2;
        gauss_lobatto_1d(n, x1, w1);
    }
    if (dim == 1) {
        for (int i = 0; i < n; ++i) { pts.insert(pts.end(), {x1[i], 0, 0}); w.push_back(w1[i]); }
    } else if (dim == 2) {
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) { pts.insert(pts.end(), {x1[j], x1[i], 0}); w.push_back(w1[i] * w1[j]); }
    } else {
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                for (int k = 0; k < n; ++k) {
                    pts.insert(pts.end(), {x1[k], x1[j], x1[i]});
                    w.push_back(w1[i] * w1[j] * w1[k]);
                }
    }
    return (int)w.size();
}

// Symmetric triangle rules on (0,0),(1,0),(0,1) of exactness 1..6: the published
// Dunavant (1985) points and weights, which the reference tabulates for
// QuadratureRule::get_triangle_quadrature (src/quadrature/TriangleQuadratureRules.cpp:9-85);
// the same values keep assembled triangle matrices identical.
int triangle_rule(int order, std::vector<double> &pts, std::vector<double> &w) {
    struct P { double x, y, w; };
    static const P r1[] = {{1. / 3., 1. / 3., 1. / 2.}};
    static const P r2[] = {{1. / 6., 1. / 6., 1. / 6.}, {1. / 6., 2. / 3., 1. / 6.}, {2. / 3., 1. / 6., 1. / 6.}};
    static const P r3[] = {{3.33333333333333333E-01, 3.33333333333333333E-01, -2.81250000000000000E-01},
                           {6.00000000000000000E-01, 2.00000000000000000E-01, 2.60416666666666667E-01},
                           {2.00000000000000000E-01, 6.00000000000000000E-01, 2.60416666666666667E-01},
                           {2.00000000000000000E-01, 2.00000000000000000E-01, 2.60416666666666666E-01}};
    static const P r4[] = {{1.081030181680700E-01, 4.459484909159650E-01, 1.116907948390055E-01},
                           {4.459484909159650E-01, 1.081030181680700E-01, 1.116907948390055E-01},
                           {4.459484909159650E-01, 4.459484909159650E-01, 1.116907948390055E-01},
                           {8.168475729804590E-01, 9.157621350977100E-02, 5.497587182766100E-02},
                           {9.157621350977100E-02, 8.168475729804590E-01, 5.497587182766100E-02},
                           {9.157621350977100E-02, 9.157621350977100E-02, 5.497587182766100E-02}};
    static const P r5[] = {{3.33333333333333E-01, 3.33333333333333E-01, 1.12500000000000E-01},
                           {5.97158717897700E-02, 4.70142064105115E-01, 6.61970763942530E-02},
                           {4.70142064105115E-01, 5.97158717897700E-02, 6.61970763942530E-02},
                           {4.70142064105115E-01, 4.70142064105115E-01, 6.61970763942530E-02},
                           {7.97426985353087E-01, 1.01286507323456E-01, 6.29695902724135E-02},
                           {1.01286507323456E-01, 7.97426985353087E-01, 6.29695902724135E-02},
                           {1.01286507323456E-01, 1.01286507323456E-01, 6.29695902724135E-02}};
    static const P r6[] = {{5.01426509658179E-01, 2.49286745170910E-01, 5.83931378631895E-02},
                           {2.49286745170910E-01, 5.01426509658179E-01, 5.83931378631895E-02},
                           {2.49286745170910E-01, 2.49286745170910E-01, 5.83931378631895E-02},
                           {8.73821971016996E-01, 6.30890144915020E-02, 2.54224531851035E-02},
                           {6.30890144915020E-02, 8.73821971016996E-01, 2.54224531851035E-02},
                           {6.30890144915020E-02, 6.30890144915020E-02, 2.54224531851035E-02},
                           {5.31450498448170E-02, 3.10352451033784E-01, 4.14255378091870E-02},
                           {6.36502499121399E-01, 5.31450498448170E-02, 4.14255378091870E-02},
                           {3.10352451033784E-01, 6.36502499121399E-01, 4.14255378091870E-02},
                           {5.31450498448170E-02, 6.36502499121399E-01, 4.14255378091870E-02},
                           {6.36502499121399E-01, 3.10352451033784E-01, 4.14255378091870E-02},
                           {3.10352451033784E-01, 5.31450498448170E-02, 4.14255378091870E-02}};
    const P *r = nullptr;
    int n = 0;
    switch (order) {
    case 1: r = r1; n = 1; break;
    case 2: r = r2; n = 3; break;
    case 3: r = r3; n = 4; break;
    case 4: r = r4; n = 6; break;
    case 5: r = r5; n = 7; break;
    case 6: r = r6; n = 12; break;
    default: return 0;
    }
    pts.clear();
    w.clear();
    for (int i = 0; i < n; ++i) { pts.insert(pts.end(), {r[i].x, r[i].y, 0.0}); w.push_back(r[i].w); }
    return n;
}

// Symmetric tetrahedron rules on (0,0,0),(1,0,0),(0,1,0),(0,0,1) of exactness
// 1..5 (Keast's published rules); the reference tabulates them with these
// digits and this point order for QuadratureRule::get_tetrahedron_quadrature
// (src/quadrature/TetrahedronQuadratureRules.cpp:27-127), and the same values
// keep assembled tetrahedron matrices identical.  Order 6 and above: none
// (the reference throws).
int tetrahedron_rule(int order, std::vector<double> &pts, std::vector<double> &w) {
    struct P { double x, y, z, w; };
    static const double a2 = 0.138196601125011, b2 = 0.585410196624969;
    static const P r1[] = {{0.25, 0.25, 0.25, 0.16666666666666666}};
    static const P r2[] = {{a2, a2, b2, 0.041666666666666664}, {a2, a2, a2, 0.041666666666666664},
                           {a2, b2, a2, 0.041666666666666664}, {b2, a2, a2, 0.041666666666666664}};
    static const double s3 = 0.16666666666666666;
    static const P r3[] = {{0.25, 0.25, 0.25, -0.13333333333333333}, {s3, 0.5, s3, 0.075}, {s3, s3, 0.5, 0.075},
                           {s3, s3, s3, 0.075}, {0.5, s3, s3, 0.075}};
    static const double a4 = 0.071428571428571, b4 = 0.785714285714286, c4 = 0.399403576166799,
                        d4 = 0.100596423833201, w4a = 0.007622222222222222, w4b = 0.024888888888888887;
    static const P r4[] = {{0.25, 0.25, 0.25, -0.013155555555555556}, {a4, a4, b4, w4a}, {a4, a4, a4, w4a},
                           {a4, b4, a4, w4a}, {b4, a4, a4, w4a}, {c4, d4, d4, w4b}, {d4, c4, c4, w4b},
                           {d4, d4, c4, w4b}, {c4, d4, c4, w4b}, {d4, c4, d4, w4b}, {c4, c4, d4, w4b}};
    static const double t5 = 0.3333333333333333, a5 = 0.09090909090909091, b5 = 0.7272727272727273,
                        c5 = 0.433449846426336, d5 = 0.066550153573664, w5a = 0.006026785714286,
                        w5b = 0.011645249086029, w5c = 0.010949141561386;
    static const P r5[] = {{0.25, 0.25, 0.25, 0.030283678097089}, {t5, t5, t5, w5a}, {0.0, t5, t5, w5a},
                           {t5, 0.0, t5, w5a}, {t5, t5, 0.0, w5a}, {a5, b5, a5, w5b}, {a5, a5, b5, w5b},
                           {a5, a5, a5, w5b}, {b5, a5, a5, w5b}, {c5, d5, c5, w5c}, {c5, c5, d5, w5c},
                           {d5, d5, c5, w5c}, {d5, c5, c5, w5c}, {c5, d5, d5, w5c}, {d5, c5, d5, w5c}};
    const P *r = nullptr;
    int n = 0;
    switch (order) {
    case 1: r = r1; n = 1; break;
    case 2: r = r2; n = 4; break;
    case 3: r = r3; n = 5; break;
    case 4: r = r4; n = 11; break;
    case 5: r = r5; n = 15; break;
    default: return 0;
    }
    pts.clear();
    w.clear();
    for (int i = 0; i < n; ++i) { pts.insert(pts.end(), {r[i].x, r[i].y, r[i].z}); w.push_back(r[i].w); }
    return n;
}

// ------------------------------------------------------------ reference elements

static double snap_to(double x, double s) { return std::round(x / s) * s; }

// Local nodes: GLL tensor product, x fastest (make_tensorproduct_element.cpp:158-193);
// triangle: Blyth-Pozrikidis warp of the GLL points snapped to 2^-21
// (make_simplex_element.cpp:17-26,94-97,156-176).
static int local_nodes(int topology, int dim, int p, std::vector<double> &pts) {
    int n = p + 1;
    double l[64], lw[64];
    gauss_lobatto_1d(n, l, lw);
    pts.clear();
    if (topology == TOPO_TENSOR || dim == 1) {
        if (dim == 1) for (int i = 0; i < n; ++i) pts.insert(pts.end(), {l[i], 0, 0});
        else if (dim == 2) for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) pts.insert(pts.end(), {l[j], l[i], 0});
        else if (dim == 3)
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j)
                    for (int k = 0; k < n; ++k) pts.insert(pts.end(), {l[k], l[j], l[i]});
        return (int)pts.size() / 3;
    }
    if (topology == TOPO_SIMPLEX && dim == 2) {
        const double snap = 1.0 / (2 << 20);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n - i; ++j) {
                int k = n - i - j - 1;
                double vi = (l[i] + 1) / 2, vj = (l[j] + 1) / 2, vk = (l[k] + 1) / 2;
                pts.insert(pts.end(), {snap_to((1 + 2 * vj - vi - vk) / 3, snap), snap_to((1 + 2 * vi - vj - vk) / 3, snap),
                                       snap_to(0.0, snap)});
            }
        return (int)pts.size() / 3;
    }
    if (topology == TOPO_SIMPLEX && dim == 3) {
        // Blyth-Pozrikidis points face by face, then interior, each coordinate
        // clipped at 0 (make_simplex_element.cpp:178-273); sorted by (z, y, x)
        // and snapped to 2^-21 as make_simplex does (:21-22,94-97)
        const double snap = 1.0 / (2 << 20);
        auto v = [&](int i) { return (l[i - 1] + 1) / 2; };
        std::vector<std::array<double, 3>> P;
        for (int i = 1; i <= n; ++i)  // xi-eta plane
            for (int j = 1; j <= n + 1 - i; ++j) {
                int k = n + 2 - i - j;
                P.push_back({std::max(0.0, (1 + 2 * v(j) - v(i) - v(k)) / 3), std::max(0.0, (1 + 2 * v(i) - v(j) - v(k)) / 3), 0.0});
            }
        for (int j = 1; j < n; ++j)  // eta-zeta plane
            for (int k = 2; k <= n + 1 - j; ++k) {
                int m = n + 2 - j - k;
                P.push_back({0.0, std::max(0.0, (1 + 2 * v(j) - v(k) - v(m)) / 3), std::max(0.0, (1 + 2 * v(k) - v(j) - v(m)) / 3)});
            }
        for (int i = 2; i < n; ++i)  // xi-zeta plane
            for (int k = 2; k <= n + 1 - i; ++k) {
                int m = n + 2 - i - k;
                P.push_back({std::max(0.0, (1 + 2 * v(i) - v(k) - v(m)) / 3), 0.0, std::max(0.0, (1 + 2 * v(k) - v(i) - v(m)) / 3)});
            }
        for (int i = 2; i < n; ++i)  // slanted face
            for (int j = 2; j <= n - i; ++j) {
                int m = n + 2 - i - j;
                const double x = std::max(0.0, (1 + 2 * v(i) - v(j) - v(m)) / 3);
                const double y = std::max(0.0, (1 + 2 * v(j) - v(i) - v(m)) / 3);
                P.push_back({x, y, 1 - x - y});
            }
        for (int i = 2; i < n; ++i)  // interior
            for (int j = 2; j <= n - i; ++j)
                for (int k = 2; k <= n + 1 - i - j; ++k) {
                    int m = n + 3 - i - j - k;
                    P.push_back({std::max(0.0, (1 + 3 * v(k) - v(i) - v(j) - v(m)) / 4),
                                 std::max(0.0, (1 + 3 * v(j) - v(i) - v(k) - v(m)) / 4),
                                 std::max(0.0, (1 + 3 * v(i) - v(j) - v(k) - v(m)) / 4)});
                }
        std::sort(P.begin(), P.end(), [](const std::array<double, 3> &a, const std::array<double, 3> &b) {
            return std::lexicographical_compare(a.rbegin(), a.rend(), b.rbegin(), b.rend());
        });
        for (auto &x : P) pts.insert(pts.end(), {snap_to(x[0], snap), snap_to(x[1], snap), snap_to(x[2], snap)});
        return (int)pts.size() / 3;
    }
    return 0;
}

// 1-D Lagrange basis on nodes x[0..n): values and derivatives at t.
static void lagrange_1d(const double *x, int n, double t, double *v, double *dv) {
    for (int j = 0; j < n; ++j) {
        double num = 1, den = 1, d = 0;
        for (int m = 0; m < n; ++m) {
            if (m == j) continue;
            den *= (x[j] - x[m]);
        }
        for (int m = 0; m < n; ++m) {
            if (m == j) continue;
            num *= (t - x[m]);
            double prod = 1;
            for (int q = 0; q < n; ++q)
                if (q != j && q != m) prod *= (t - x[q]);
            d += prod;
        }
        v[j] = num / den;
        dv[j] = d / den;
    }
}

// Dense LU with partial pivoting (row-major, in place) and solve.
static void lu_factor(std::vector<double> &A, int n, std::vector<int> &piv) {
    piv.resize(n);
    std::iota(piv.begin(), piv.end(), 0);
    for (int k = 0; k < n; ++k) {
        int p = k;
        for (int i = k + 1; i < n; ++i)
            if (std::fabs(A[i * n + k]) > std::fabs(A[p * n + k])) p = i;
        if (p != k) {
            for (int j = 0; j < n; ++j) std::swap(A[k * n + j], A[p * n + j]);
            std::swap(piv[k], piv[p]);
        }
        for (int i = k + 1; i < n; ++i) {
            A[i * n + k] /= A[k * n + k];
            for (int j = k + 1; j < n; ++j) A[i * n + j] -= A[i * n + k] * A[k * n + j];
        }
    }
}
static void lu_solve(const std::vector<double> &LU, int n, const std::vector<int> &piv, const double *b, double *x) {
    std::vector<double> y(n);
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

// Forward-mode dual number (value, derivative).
struct Dual {
    double f, d;
};
static Dual operator+(Dual a, Dual b) { return {a.f + b.f, a.d + b.d}; }
static Dual operator-(Dual a, Dual b) { return {a.f - b.f, a.d - b.d}; }
static Dual operator*(Dual a, Dual b) { return {a.f * b.f, a.d * b.f + a.f * b.d}; }
static Dual operator/(Dual a, Dual b) { return {a.f / b.f, (a.d * b.f - a.f * b.d) / (b.f * b.f)}; }
static Dual dpow(Dual x, int e) { return {std::pow(x.f, e), x.d * e * std::pow(x.f, e - 1)}; }

// Jacobi polynomial P_n^{(a,b)} coefficients, highest degree first, by the
// three-term recurrence (the reference's jacobi(), ShapeFunctionUtils.cpp:16-62).
static std::vector<double> jacobi_coeffs(int n, double a, double b) {
    std::vector<double> c1{(a + b + 2) / 2, (a - b) / 2}, c2{1.0};
    if (n == 0) return c2;
    if (n == 1) return c1;
    std::vector<double> c = c1;
    for (int i = 1; i < n; ++i) {
        double tmp = i + a + b + 1;
        double A = (2 * i + a + b + 1) * (2 * i + a + b + 2) / (2 * (i + 1) * tmp);
        double B = (b * b - a * a) * (2 * i + a + b + 1) / (2 * (i + 1) * tmp * (2 * i + a + b));
        double Cc = (i + a) * (i + b) * (2 * i + a + b + 2) / ((i + 1) * tmp * (2 * i + a + b));
        c.push_back(0);
        for (double &v : c) v *= A;
        for (size_t k = 0; k < c1.size(); ++k) c[c.size() - 1 - k] -= B * c1[c1.size() - 1 - k];
        for (size_t k = 0; k < c2.size(); ++k) c[c.size() - 1 - k] -= Cc * c2[c2.size() - 1 - k];
        c2 = c1;
        c1 = c;
    }
    return c;
}

static Dual horner(const std::vector<double> &c, Dual x) {
    Dual r{0, 0};
    for (double v : c) r = r * x + Dual{v, 0};
    return r;
}

// Koornwinder basis on the triangle, phi_k = P_m(r) P_n^{(2m+1,0)}(s) ((1-s)/2)^m
// with r = 2(1+xi)/(1-eta) - 1, s = eta, (m,n) ordered as the reference orders
// them (ShapeFunctionUtils.cpp:160-189).  g selects the derivative direction
// (-1: value only).
struct Koornwinder {
    int p;
    std::vector<std::vector<double>> j00;
    std::vector<int> m;
    std::vector<std::vector<double>> j2;
    explicit Koornwinder(int p_) : p(p_) {
        for (int k = 0; k <= p; ++k) j00.push_back(jacobi_coeffs(k, 0, 0));
        for (int i = 0; i <= p; ++i)
            for (int j = 0; j <= p; ++j)
                if (i + j <= p) {
                    m.push_back(i);
                    j2.push_back(jacobi_coeffs(j, 2 * i + 1, 0));
                }
    }
    Dual eval(int k, double x, double y, int g) const {
        Dual xi{x, g == 0 ? 1.0 : 0.0}, eta{y, g == 1 ? 1.0 : 0.0};
        Dual one{1, 0}, two{2, 0};
        Dual r = two * (one + xi) / (one - eta) - one;
        Dual s = eta;
        return horner(j00[m[k]], r) * horner(j2[k], s) * dpow((one - s) / two, m[k]);
    }
};

// The reference's orthogonal basis on the tetrahedron,
// phi_k = P_m(r) P_n^{(2m+1,0)}(s) P_l^{(2m+2n+2,0)}(t) ((1-s)/2)^m ((1-t)/2)^(m+n)
// with r = -2(1+xi)/(eta+zeta) - 1, s = 2(1+eta)/(1-zeta) - 1, t = zeta and
// (m,n,l) in the reference's loop order (ShapeFunctionUtils.cpp:230-281).
struct TetBasis {
    std::vector<std::vector<double>> j00, j2, j3;
    std::vector<int> m, n;
    explicit TetBasis(int p) {
        for (int k = 0; k <= p; ++k) j00.push_back(jacobi_coeffs(k, 0, 0));
        for (int i = 0; i <= p; ++i)
            for (int j = 0; j <= p; ++j)
                for (int k = 0; k <= p; ++k)
                    if (i + j + k <= p) {
                        m.push_back(i);
                        n.push_back(j);
                        j2.push_back(jacobi_coeffs(j, 2 * i + 1, 0));
                        j3.push_back(jacobi_coeffs(k, 2 * i + 2 * j + 2, 0));
                    }
    }
    Dual eval(int k, double x, double y, double z, int g) const {
        Dual xi{x, g == 0 ? 1.0 : 0.0}, eta{y, g == 1 ? 1.0 : 0.0}, zeta{z, g == 2 ? 1.0 : 0.0};
        Dual one{1, 0}, two{2, 0};
        Dual r = Dual{-2, 0} * (one + xi) / (eta + zeta) - one;
        Dual s = two * (one + eta) / (one - zeta) - one;
        Dual t = zeta;
        return horner(j00[m[k]], r) * horner(j2[k], s) * horner(j3[k], t) * dpow((one - s) / two, m[k]) *
               dpow((one - t) / two, m[k] + n[k]);
    }
};

bool make_element_table(int topology, int dim, int p, ElementTable &T) {
    T.topology = topology;
    T.dim = dim;
    T.p = p;
    T.nen = local_nodes(topology, dim, p, T.local_nodes);
    if (T.nen <= 0) return false;
    if (topology == TOPO_TENSOR || dim == 1) {
        // volume rule: Gauss-Legendre of exactness 2p (make_tensorproduct_element.cpp:127-128)
        T.nq = tensor_rule(false, dim, 2 * p, T.qpts, T.qw);
        // tensor-product Lagrange basis on the GLL points; node A = (i,j,k), x fastest
        const int n = p + 1;
        double l[64], lw[64];
        gauss_lobatto_1d(n, l, lw);
        T.N.assign((size_t)T.nq * T.nen, 0.0);
        T.dN.assign((size_t)T.nq * T.nen * dim, 0.0);
        for (int q = 0; q < T.nq; ++q) {
            double v[3][64], dv[3][64];
            for (int d = 0; d < dim; ++d) lagrange_1d(l, n, T.qpts[3 * q + d], v[d], dv[d]);
            for (int A = 0; A < T.nen; ++A) {
                int idx[3] = {A % n, (A / n) % n, A / (n * n)};
                double val = 1;
                for (int d = 0; d < dim; ++d) val *= v[d][idx[d]];
                T.N[(size_t)q * T.nen + A] = val;
                for (int g = 0; g < dim; ++g) {
                    double dval = 1;
                    for (int d = 0; d < dim; ++d) dval *= (d == g) ? dv[d][idx[d]] : v[d][idx[d]];
                    T.dN[((size_t)q * T.nen + A) * dim + g] = dval;
                }
            }
        }
        return true;
    }
    if (topology == TOPO_SIMPLEX && dim == 2) {
        // volume rule of exactness 2p (make_simplex_element.cpp:99-100)
        T.nq = triangle_rule(std::max(1, 2 * p), T.qpts, T.qw);
        if (T.nq == 0) return false;
        // Nodal basis from the Koornwinder Vandermonde V(i,j) = phi_j(x_i) on the
        // node set whose top vertex sits at y = 0.999999999, solved as V^T N = phi(xi)
        // with partial-pivot LU and dual-number gradients -- the reference's
        // construction (ShapeFunctionUtils.cpp:145-217), so the rounding matches.
        const int nen = T.nen;
        std::vector<double> nodes = T.local_nodes;
        for (int i = 0; i < nen; ++i) nodes[3 * i + 1] = std::min(.999999999, nodes[3 * i + 1]);
        Koornwinder K(p);
        std::vector<double> VT((size_t)nen * nen);
        for (int i = 0; i < nen; ++i)
            for (int j = 0; j < nen; ++j) VT[(size_t)j * nen + i] = K.eval(j, nodes[3 * i], nodes[3 * i + 1], -1).f;
        std::vector<int> piv;
        lu_factor(VT, nen, piv);
        T.N.assign((size_t)T.nq * nen, 0.0);
        T.dN.assign((size_t)T.nq * nen * 2, 0.0);
        std::vector<double> v(nen), dx(nen), dy(nen), sol(nen);
        for (int q = 0; q < T.nq; ++q) {
            const double x = T.qpts[3 * q], y = T.qpts[3 * q + 1];
            for (int j = 0; j < nen; ++j) {
                v[j] = K.eval(j, x, y, -1).f;
                dx[j] = K.eval(j, x, y, 0).d;
                dy[j] = K.eval(j, x, y, 1).d;
            }
            lu_solve(VT, nen, piv, v.data(), sol.data());
            for (int A = 0; A < nen; ++A) T.N[(size_t)q * nen + A] = sol[A];
            lu_solve(VT, nen, piv, dx.data(), sol.data());
            for (int A = 0; A < nen; ++A) T.dN[((size_t)q * nen + A) * 2 + 0] = sol[A];
            lu_solve(VT, nen, piv, dy.data(), sol.data());
            for (int A = 0; A < nen; ++A) T.dN[((size_t)q * nen + A) * 2 + 1] = sol[A];
        }
        return true;
    }
    if (topology == TOPO_SIMPLEX && dim == 3) {
        // volume rule of exactness 2p (make_simplex_element.cpp:101-103); the
        // reference has rules up to exactness 5, so p <= 2
        T.nq = tetrahedron_rule(std::max(1, 2 * p), T.qpts, T.qw);
        if (T.nq == 0) return false;
        // nodal basis from the Vandermonde of TetBasis on the node set with
        // zeta capped at 0.999999999 and points on the eta = zeta = 0 edge moved
        // by 1e-8 in eta and zeta (ShapeFunctionUtils.cpp:220-304)
        const int nen = T.nen;
        std::vector<double> nodes = T.local_nodes;
        for (int i = 0; i < nen; ++i) {
            nodes[3 * i + 2] = std::min(.999999999, nodes[3 * i + 2]);
            if (nodes[3 * i + 1] + nodes[3 * i + 2] == 0) {
                nodes[3 * i + 1] += 0.00000001;
                nodes[3 * i + 2] += 0.00000001;
            }
        }
        TetBasis K(p);
        std::vector<double> VT((size_t)nen * nen);
        for (int i = 0; i < nen; ++i)
            for (int j = 0; j < nen; ++j)
                VT[(size_t)j * nen + i] = K.eval(j, nodes[3 * i], nodes[3 * i + 1], nodes[3 * i + 2], -1).f;
        std::vector<int> piv;
        lu_factor(VT, nen, piv);
        T.N.assign((size_t)T.nq * nen, 0.0);
        T.dN.assign((size_t)T.nq * nen * 3, 0.0);
        std::vector<double> v(nen), dg(nen), sol(nen);
        for (int q = 0; q < T.nq; ++q) {
            const double x = T.qpts[3 * q], y = T.qpts[3 * q + 1], z = T.qpts[3 * q + 2];
            for (int j = 0; j < nen; ++j) v[j] = K.eval(j, x, y, z, -1).f;
            lu_solve(VT, nen, piv, v.data(), sol.data());
            for (int A = 0; A < nen; ++A) T.N[(size_t)q * nen + A] = sol[A];
            for (int g = 0; g < 3; ++g) {
                for (int j = 0; j < nen; ++j) dg[j] = K.eval(j, x, y, z, g).d;
                lu_solve(VT, nen, piv, dg.data(), sol.data());
                for (int A = 0; A < nen; ++A) T.dN[((size_t)q * nen + A) * 3 + g] = sol[A];
            }
        }
        return true;
    }
    return false;
}

// ------------------------------------------------------------ DoF numbering

void cell_element_type(int ct, int &topo, int &tdim) {
    switch (ct) {
    case CELL_LINE2: topo = TOPO_TENSOR; tdim = 1; break;
    case CELL_TRI3: topo = TOPO_SIMPLEX; tdim = 2; break;
    case CELL_TET4: topo = TOPO_SIMPLEX; tdim = 3; break;
    case CELL_QUAD4: topo = TOPO_TENSOR; tdim = 2; break;
    case CELL_HEX8: topo = TOPO_TENSOR; tdim = 3; break;
    default: topo = TOPO_NONE; tdim = 0; break;
    }
}

// DoFManager::interpolate_from_corners (src/utils/DoFManager.cpp:296-338), with
// the reference's operation order so the merged node set is the same.
static void interpolate_from_corners(const double *xl, const double *c, int ct, double *out) {
    const double x0 = xl[0], x1 = xl[1], x2 = xl[2];
    for (int k = 0; k < 3; ++k) {
        switch (ct) {
        case CELL_TRI3: out[k] = (1 - x0 - x1) * c[k] + x0 * c[3 + k] + x1 * c[6 + k]; break;
        case CELL_TET4: out[k] = (1 - x0 - x1 - x2) * c[k] + x0 * c[3 + k] + x1 * c[6 + k] + x2 * c[9 + k]; break;
        case CELL_QUAD4:
            out[k] = (1.0 / 4.0) * ((1 - x0) * (1 - x1) * c[k] + (1 + x0) * (1 - x1) * c[3 + k] +
                                    (1 + x0) * (1 + x1) * c[6 + k] + (1 - x0) * (1 + x1) * c[9 + k]);
            break;
        case CELL_HEX8:
            out[k] = (1.0 / 8.0) * ((1 - x0) * (1 - x1) * (1 - x2) * c[k] + (1 + x0) * (1 - x1) * (1 - x2) * c[3 + k] +
                                    (1 + x0) * (1 + x1) * (1 - x2) * c[6 + k] + (1 - x0) * (1 + x1) * (1 - x2) * c[9 + k] +
                                    (1 - x0) * (1 - x1) * (1 + x2) * c[12 + k] + (1 + x0) * (1 - x1) * (1 + x2) * c[15 + k] +
                                    (1 + x0) * (1 + x1) * (1 + x2) * c[18 + k] + (1 - x0) * (1 + x1) * (1 + x2) * c[21 + k]);
            break;
        default: out[k] = 0; break;
        }
    }
}

// Stable LSD radix sort of the N keys `ka` (only the low `nbits` bits are set;
// the array is used as scratch) into the permutation `out_idx` (out_idx[j] =
// position of the j-th smallest key; equal keys keep their original order).  11-bit digits; each pass counts per thread and
// scatters each thread's contiguous chunk in order, so the result does not
// depend on the thread count.
static void radix_sort_index(uint64_t *ka, int64_t N, int nbits, int64_t *out_idx) {
    constexpr int D = 11, R = 1 << D;
    std::unique_ptr<uint64_t[]> kb(new uint64_t[N]);
    std::unique_ptr<int64_t[]> ia_buf(new int64_t[N]), ib_buf(new int64_t[N]);
    uint64_t *kin = ka, *kout = kb.get();
    int64_t *iin = ia_buf.get(), *iout = ib_buf.get();
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) iin[i] = i;
    int T = 1;
#ifdef _OPENMP
    T = omp_get_max_threads();
#endif
    std::vector<int64_t> hist((size_t)T * R);
    for (int shift = 0; shift < nbits; shift += D) {
        std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(T)
        {
            int t = 0;
#ifdef _OPENMP
            t = omp_get_thread_num();
#endif
            const int64_t lo = N * t / T, hi = N * (t + 1) / T;
            int64_t *h = &hist[(size_t)t * R];
            for (int64_t i = lo; i < hi; ++i) ++h[(kin[i] >> shift) & (R - 1)];
#pragma omp barrier
#pragma omp single
            {
                int64_t sum = 0;
                for (int q = 0; q < R; ++q)
                    for (int u = 0; u < T; ++u) {
                        int64_t c = hist[(size_t)u * R + q];
                        hist[(size_t)u * R + q] = sum;
                        sum += c;
                    }
            }
            for (int64_t i = lo; i < hi; ++i) {
                const int64_t dst = h[(kin[i] >> shift) & (R - 1)]++;
                kout[dst] = kin[i];
                iout[dst] = iin[i];
            }
        }
        std::swap(kin, kout);
        std::swap(iin, iout);
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) out_idx[i] = iin[i];
}

int64_t raw_node_layout(int32_t n_cells, int32_t p, HostDofmap &d, RawLayout &lay) {
    int64_t offset = 0;
    for (int c = 0; c < n_cells; ++c) {
        const int t = d.topology[c], td = d.topo_dim[c];
        d.offsets[c] = (int32_t)offset;
        if (t == TOPO_NONE) continue;
        if (!lay.nloc[t][td]) lay.nloc[t][td] = local_nodes(t, td, p, lay.loc[t][td]);
        offset += lay.nloc[t][td];
    }
    d.offsets[n_cells] = (int32_t)offset;
    return offset;
}

bool raw_mix_needs_reference_order(const HostDofmap &d, int64_t n_raw) {
    bool has_simplex = false, has_tensor = false;
    for (int32_t c = 0; c < d.n_cells(); ++c) {
        has_simplex |= d.topology[c] == TOPO_SIMPLEX && d.topo_dim[c] >= 2;
        has_tensor |= d.topology[c] == TOPO_TENSOR && d.topo_dim[c] >= 2;
    }
    return n_raw <= kReferenceOrderMaxRawNodes || (d.poly_order >= 3 && has_simplex && has_tensor);
}

bool build_dofmap(const double *xyz, int32_t n_nodes, const int32_t *cell_nodes, const int32_t *cell_offsets,
                  const int32_t *cell_types, int32_t n_cells, int32_t p, int32_t dpn, HostDofmap &d) {
    if (p < 1) return false;
    d.dof_per_node = dpn;
    d.poly_order = p;
    d.offsets.assign(n_cells + 1, 0);
    d.topology.resize(n_cells);
    d.topo_dim.resize(n_cells);
    d.porder.assign(n_cells, (int8_t)p);
    for (int c = 0; c < n_cells; ++c) {
        int t, td;
        cell_element_type(cell_types[c], t, td);
        d.topology[c] = (int8_t)t;
        d.topo_dim[c] = (int8_t)td;
    }
    if (p == 1) {  // DoFManager.cpp:153-160
        d.nodes.assign(xyz, xyz + 3 * (int64_t)n_nodes);
        d.offsets.assign(cell_offsets, cell_offsets + n_cells + 1);
        d.elements.assign(cell_nodes, cell_nodes + cell_offsets[n_cells]);
        return true;
    }
    // make_raw_dofs (DoFManager.cpp:176-229): every element's nodes at the
    // element's local node coordinates, cells in mesh order (offsets first, then
    // the coordinates of all cells in parallel)
    RawLayout lay;
    const int64_t N = raw_node_layout(n_cells, p, d, lay);
    const auto &tabs = lay.loc;
    const auto &nloc = lay.nloc;
    std::unique_ptr<double[]> raw(new double[3 * N]);  // written (first touched) in parallel below
#pragma omp parallel for schedule(static)
    for (int c = 0; c < n_cells; ++c) {
        int t = d.topology[c], td = d.topo_dim[c];
        if (t == TOPO_NONE) continue;
        const std::vector<double> &L = tabs[t][td];
        const int nl = nloc[t][td];
        double corners[24] = {0};
        int nc = cell_offsets[c + 1] - cell_offsets[c];
        for (int i = 0; i < nc && i < 8; ++i)
            for (int k = 0; k < 3; ++k) corners[3 * i + k] = xyz[3 * (int64_t)cell_nodes[cell_offsets[c] + i] + k];
        double *o = &raw[3 * (int64_t)d.offsets[c]];
        for (int a = 0; a < nl; ++a) interpolate_from_corners(&L[3 * a], corners, cell_types[c], o + 3 * a);
    }
    // recombine_all_duplicates (DoFManager.cpp:340-414): sort on the snapped
    // coordinates (z, y, x), merge neighbours closer than 1e-6.  The snapped value
    // is k*s with k = round(x/s) an integer, so the order of the snapped doubles is
    // the order of the integer triples, which pack into one 64-bit key; a stable
    // sort keeps equal keys in raw order, as a (key, index) sort does.
    if (N == 0) { d.nodes.clear(); return true; }
    double bmin[3] = {raw[0], raw[1], raw[2]}, bmax[3] = {raw[0], raw[1], raw[2]};
    for (int k = 0; k < 3; ++k) {
        double lo = raw[k], hi = raw[k];
#pragma omp parallel for reduction(min : lo) reduction(max : hi) schedule(static)
        for (int64_t i = 0; i < N; ++i) {
            lo = std::min(lo, raw[3 * i + k]);
            hi = std::max(hi, raw[3 * i + k]);
        }
        bmin[k] = lo;
        bmax[k] = hi;
    }
    double max_dim = std::max(bmax[0] - bmin[0], std::max(bmax[1] - bmin[1], bmax[2] - bmin[2]));
    double snapv = max_dim * 1.0e-6;
    // snapped integer coordinates: ranges first, keys second (nothing stored).
    // The reference's tensor division by a scalar multiplies by its reciprocal
    // (lin_alg/tensor/tensor_functions/operators.hpp:66-70), so the key is
    // round(x * (1/s)); a true division would round differently near .5.
    const double inv_snap = snapv > 0 ? 1.0 / snapv : 0.0;
    auto snapped = [&](int64_t i, int k) -> int64_t {
        return (snapv > 0) ? (int64_t)std::llround(std::round(raw[3 * i + k] * inv_snap)) : 0;
    };
    int64_t kmin[3], kmax[3];
    for (int k = 0; k < 3; ++k) {
        int64_t lo = INT64_MAX, hi = INT64_MIN;
#pragma omp parallel for reduction(min : lo) reduction(max : hi) schedule(static)
        for (int64_t i = 0; i < N; ++i) {
            const int64_t v = snapped(i, k);
            lo = std::min(lo, v);
            hi = std::max(hi, v);
        }
        kmin[k] = lo;
        kmax[k] = hi;
    }
    int bits[3];
    for (int k = 0; k < 3; ++k) {
        const uint64_t span = (uint64_t)(kmax[k] - kmin[k]);
        bits[k] = 0;
        while (bits[k] < 63 && (span >> bits[k]) != 0) ++bits[k];
    }
    const bool packable = bits[0] + bits[1] + bits[2] <= 64;
    std::unique_ptr<int64_t[]> idx(new int64_t[N]);
    // Which of several coincident raw nodes gives the merged node its
    // coordinates is the first one in sorted order.  The reference sorts with
    // std::sort on the snapped key alone (DoFManager.cpp:371), an unstable sort,
    // so among equal keys its order is whatever std::sort produces.  Coincident
    // raw nodes usually differ only in rounding, but where triangles (whose
    // local nodes are snapped to 2^-21, make_simplex_element.cpp:21-22,94-97)
    // meet quadrilaterals at p >= 3 they differ by up to 2.4e-7 of the cell
    // size, and the choice changes the geometry.  Small meshes, and every mesh
    // that mixes simplex and tensor cells at p >= 3, are therefore sorted with
    // std::sort and the reference's comparison (no tie-break) from the same
    // identity permutation, which reproduces its order exactly; large meshes
    // use the stable parallel radix sort (same node numbering; merged
    // coordinates can differ from the reference's in the last bit).
    const bool reference_order = raw_mix_needs_reference_order(d, N);
    if (reference_order) {
        std::vector<int64_t> kq(3 * N);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i)
            for (int k = 0; k < 3; ++k) kq[3 * i + k] = snapped(i, k);
        std::vector<int32_t> ids(N);
        std::iota(ids.begin(), ids.end(), 0);
        std::sort(ids.begin(), ids.end(), [&](int32_t a, int32_t b) {
            for (int k = 2; k >= 0; --k)
                if (kq[3 * (int64_t)a + k] != kq[3 * (int64_t)b + k]) return kq[3 * (int64_t)a + k] < kq[3 * (int64_t)b + k];
            return false;
        });
        for (int64_t i = 0; i < N; ++i) idx[i] = ids[i];
    } else if (packable) {
        std::unique_ptr<uint64_t[]> keys(new uint64_t[N]);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i)
            keys[i] = ((uint64_t)(snapped(i, 2) - kmin[2]) << (bits[0] + bits[1])) |
                      ((uint64_t)(snapped(i, 1) - kmin[1]) << bits[0]) | (uint64_t)(snapped(i, 0) - kmin[0]);
        radix_sort_index(keys.get(), N, bits[0] + bits[1] + bits[2], idx.get());
    } else {
        std::vector<int64_t> kq(3 * N);
        for (int64_t i = 0; i < N; ++i)
            for (int k = 0; k < 3; ++k) kq[3 * i + k] = snapped(i, k);
        std::iota(idx.get(), idx.get() + N, 0);
        std::sort(idx.get(), idx.get() + N, [&](int64_t a, int64_t b) {
            for (int k = 2; k >= 0; --k)
                if (kq[3 * a + k] != kq[3 * b + k]) return kq[3 * a + k] < kq[3 * b + k];
            return a < b;
        });
    }
    // merge: a sorted entry starts a new node unless it lies within 1e-6 of the
    // previous one; node numbers are the running count of starts
    std::unique_ptr<int32_t[]> start(new int32_t[N]);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) {
        int32_t newg = 1;
        if (i > 0) {
            const double *a = &raw[3 * idx[i]], *b = &raw[3 * idx[i - 1]];
            double s2 = 0;
            for (int k = 0; k < 3; ++k) s2 += (a[k] - b[k]) * (a[k] - b[k]);
            if (std::sqrt(s2) < 1.0e-6) newg = 0;
        }
        start[i] = newg;
    }
    std::vector<int64_t> first;
    first.reserve(N / 2 + 1);
    for (int64_t i = 0; i < N; ++i) {
        if (start[i]) first.push_back(idx[i]);
        start[i] = (int32_t)(first.size() - 1);  // now the node number of sorted entry i
    }
    d.elements.resize(N);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) d.elements[idx[i]] = start[i];
    d.nodes.resize(3 * first.size());
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < (int64_t)first.size(); ++g)
        for (int k = 0; k < 3; ++k) d.nodes[3 * g + k] = raw[3 * first[g] + k];
    return true;
}

int color_cells(const HostDofmap &d, int nsd, int topology, std::vector<int32_t> &order, std::vector<int32_t> &ptr) {
    const int32_t nc = d.n_cells();
    std::vector<uint64_t> used(d.n_nodes(), 0);
    std::vector<int8_t> color(nc, -1);
    int ncolors = 0;
    for (int32_t c = 0; c < nc; ++c) {
        if (d.topo_dim[c] != nsd || d.topology[c] != topology) continue;
        uint64_t mask = 0;
        for (int32_t i = d.offsets[c]; i < d.offsets[c + 1]; ++i) mask |= used[d.elements[i]];
        int col = 0;
        while (col < 64 && (mask >> col) & 1) ++col;
        if (col == 64) return -1;
        color[c] = (int8_t)col;
        for (int32_t i = d.offsets[c]; i < d.offsets[c + 1]; ++i) used[d.elements[i]] |= (uint64_t(1) << col);
        ncolors = std::max(ncolors, col + 1);
    }
    ptr.assign(ncolors + 1, 0);
    for (int32_t c = 0; c < nc; ++c)
        if (color[c] >= 0) ptr[color[c] + 1]++;
    for (int k = 0; k < ncolors; ++k) ptr[k + 1] += ptr[k];
    order.resize(ptr[ncolors]);
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
    for (int32_t c = 0; c < nc; ++c)
        if (color[c] >= 0) order[fill[color[c]]++] = c;
    return ncolors;
}

}  // namespace yg
