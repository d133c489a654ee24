/*
 * ORACLE — test infrastructure only (see oracle2d.h). Never part of the
 * product path; the product library fails loudly if its CUDA code is missing
 * and has no CPU fallback.
 *
 * FP64 restatement of the reference's 2-D field-mode tracer. Function-level
 * citations are "file:line" relative to the reference project root. Floating
 * point operation order follows the reference (vector helpers follow the GLM
 * API definitions: dot = x*x' + y*y', length = sqrt(dot)), literals marked
 * FL() in the reference are float literals and are reproduced as (double)Xf.
 * Complex arithmetic uses C99 complex, which GCC lowers exactly as libstdc++
 * lowers std::complex<double>.
 */
#include "oracle2d.h"

#include <complex.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cpx;
typedef struct { double x, y; } v2;

#define PI 3.14159265358979323846
#define FLT(x) ((double)(x##f))
#define REAL_EPS DBL_EPSILON
#define INF_STEP 1e-6      /* src/step.hpp:28-32 */
#define MAXN 100000        /* include/bhc/structs.hpp:66 */
#define RAD_DEG (180.0 / PI)
#define DEG_RAD (PI / 180.0)

/* error / warning codes: src/util/errors.hpp:61-93 */
enum { E_TEMPLATE = 0, E_RAYINIT = 2, E_BDRY_NAN = 3, E_BC_TYPE = 4, E_SSP_TYPE = 5,
       E_OUT_ALT = 6, E_OUT_BTY = 7 };
enum { W_ONERAY_MEM = 1, W_TOO_FEW = 3, W_SRC_OUTSIDE = 4, W_STEP_NEG = 8,
       W_PCHIP_XT = 16, W_PCHIP_COEF = 17 };

static inline v2 V(double x, double y) { v2 r = {x, y}; return r; }
static inline v2 vadd(v2 a, v2 b) { return V(a.x + b.x, a.y + b.y); }
static inline v2 vsub(v2 a, v2 b) { return V(a.x - b.x, a.y - b.y); }
static inline v2 vsc(double s, v2 a) { return V(s * a.x, s * a.y); }
static inline v2 vdiv(v2 a, double s) { return V(a.x / s, a.y / s); }
static inline double vdot(v2 a, v2 b) { return a.x * b.x + a.y * b.y; }
static inline double vlen(v2 a) { return sqrt(vdot(a, a)); }
static inline double dmin(double a, double b) { return (b < a) ? b : a; }
static inline double dmax(double a, double b) { return (a < b) ? b : a; }
static inline int imin(int a, int b) { return (b < a) ? b : a; }
static inline int imax(int a, int b) { return (a < b) ? b : a; }
/* src/common.hpp:246-250 */
static inline double spacing(double v) { return fabs(nextafter(v, 0.0) - v); }

/* ------------------------------------------------------------------ */
/* environment after preprocessing                                      */
/* ------------------------------------------------------------------ */
typedef struct { cpx cP, cS; double rho; char bc; } HS;

typedef struct {
    v2 x, t, n, Nodet, Noden;
    double Len, Dx, Dxx, Dss, kappa;
    HS hs;
} BdPt; /* include/bhc/structs.hpp:147-170 (2-D members) */

typedef struct {
    int n;
    char type[2];
    BdPt *bd;
} Bdry;

typedef struct {
    /* SSP tables (include/bhc/structs.hpp:73-91) */
    char type;
    int npts;
    double *z, *rho;
    cpx *c, *cz, *n2, *n2z, *spl[4], *coef[4];
    /* halfspaces */
    HS top, bot;
    double top_depth, bot_depth;
    Bdry btop, bbot;
    /* positions */
    int nsz, nrz, nrr, nrz_per_range;
    float *sz, *rz;
    double *rr, delta_r;
    /* angles */
    int nalpha, isingle;
    double *alpha, dalpha;
    /* beam */
    char run_type[7], beam_type[4];
    double deltas, box_x, box_y;
    double freq0;
    int nsbp;
    double *sbp;
    /* outputs */
    int max_narr, allow_merging, eigen_memsize;
} Env;

typedef struct { unsigned err, warn; } ErrSt;
static void run_error(ErrSt *e, int c) { e->err |= 1u << c; }
static void run_warn(ErrSt *e, int c) { e->warn |= 1u << c; }

/* ------------------------------------------------------------------ */
/* host preprocessing                                                   */
/* ------------------------------------------------------------------ */

/* src/module/atten.cpp:40-70 */
static double franc_garr(double f, const O2Env *a)
{
    double c, a1, a2, a3, p1, p2, p3, f1, f2;
    c = FLT(1412.0) + FLT(3.21) * a->fg_T + FLT(1.19) * a->fg_S + FLT(0.0167) * a->fg_zbar;
    a1 = FLT(8.86) / c * pow(FLT(10.0), FLT(0.78) * a->fg_pH - FLT(5.0));
    p1 = FLT(1.0);
    f1 = FLT(2.8) * sqrt(a->fg_S / 35) * pow(FLT(1.0), FLT(4.0) - FLT(1245.0) / (a->fg_T + FLT(273.0)));
    a2 = FLT(21.44) * a->fg_S / c * (FLT(1.0) + FLT(0.025) * a->fg_T);
    p2 = FLT(1.0) - 1.37e-4 * a->fg_zbar + 6.2e-9 * a->fg_zbar * a->fg_zbar;
    f2 = FLT(8.17) * pow(FLT(10.0), FLT(8.0) - FLT(1990.0) / (a->fg_T + 273))
        / (FLT(1.0) + FLT(0.0018) * (a->fg_S - FLT(35.0)));
    p3 = FLT(1.0) - 3.83e-5 * a->fg_zbar + 4.9e-10 * a->fg_zbar * a->fg_zbar;
    double t = a->fg_T;
    if(t < FLT(20.0))
        a3 = 4.937e-4 - 2.59e-5 * t + 9.11e-7 * t * t - 1.5e-8 * t * t * t;
    else
        a3 = 3.964e-4 - 1.146e-5 * t + 1.45e-7 * t * t - 6.5e-10 * t * t * t;
    return a1 * p1 * (f1 * f * f) / (f1 * f1 + f * f) + a2 * p2 * (f2 * f * f) / (f2 * f2 + f * f)
        + a3 * p3 * f * f;
}

/* src/module/atten.cpp:99-194 (crci); fT is 1e20 unless an 'A' halfspace was read */
static cpx crci(const O2Env *env, double fT, double z, double c, double alpha, const char au[2])
{
    double freq = env->freq0, freq0 = env->freq0;
    double omega = FLT(2.0) * PI * freq;
    double alphaT = FLT(0.0);
    switch(au[0]) {
    case 'N': alphaT = alpha; break;
    case 'M': alphaT = alpha / 8.6858896; break;
    case 'm':
        alphaT = alpha / 8.6858896;
        if(freq < fT) alphaT *= pow(freq / freq0, 1.0);
        else alphaT *= (freq / freq0) * pow(fT / freq0, 1.0 - FLT(1.0));
        break;
    case 'F': alphaT = alpha * freq / 8685.8896; break;
    case 'W':
        if(fabs(c) >= REAL_EPS) alphaT = alpha * freq / (8.6858896 * c);
        break;
    case 'Q':
        if(fabs(c * alpha) >= REAL_EPS) alphaT = omega / (FLT(2.0) * c * alpha);
        break;
    case 'L':
        if(fabs(c) >= REAL_EPS) alphaT = alpha * omega / c;
        break;
    }
    switch(au[1]) {
    case 'T': {
        double f2 = (freq / FLT(1000.0)) * (freq / FLT(1000.0));
        double Thorp = FLT(3.3e-3) + FLT(0.11) * f2 / (FLT(1.0) + f2)
            + FLT(44.0) * f2 / (FLT(4100.0) + f2) + FLT(3e-4) * f2;
        Thorp /= FLT(8685.8896);
        alphaT += Thorp;
    } break;
    case 'F': {
        double fg = franc_garr(freq / FLT(1000.0), env);
        fg /= FLT(8685.8896);
        alphaT += fg;
    } break;
    case 'B':
        for(int i = 0; i < env->nbio; ++i) {
            const double *b = env->bio + 5 * i;
            if(z >= b[0] && z <= b[1]) {
                double q = 1.0 - (b[2] * b[2]) / (freq * freq);
                double a = b[4] / (q * q + 1.0 / (b[3] * b[3]));
                a /= FLT(8685.8896);
                alphaT += a;
            }
        }
        break;
    }
    alphaT *= (c * c) / omega;
    return CMPLX(c, alphaT);
}

/* src/module/boundarycond.hpp:171-224 */
static HS make_hs(const O2Env *env, double fT, char bc, const double *h)
{
    HS hs;
    memset(&hs, 0, sizeof(hs));
    hs.bc = bc;
    if(bc == 'A') {
        hs.cP = crci(env, fT, h[0], h[1], h[4], env->atten_unit);
        hs.cS = crci(env, fT, h[0], h[2], h[5], env->atten_unit);
        hs.rho = h[3];
    } else if(bc == 'G') {
        double Mz = h[6], vr, alpha2_f;
        if(Mz >= FLT(-1.0) && Mz < FLT(1.0)) {
            vr = FLT(0.002709) * Mz * Mz - FLT(0.056452) * Mz + FLT(1.2778);
            hs.rho = FLT(0.007797) * Mz * Mz - FLT(0.17057) * Mz + FLT(2.3139);
        } else if(Mz >= FLT(1.0) && Mz < FLT(5.3)) {
            vr = FLT(-0.0014881) * Mz * Mz * Mz + FLT(0.0213937) * Mz * Mz - FLT(0.1382798) * Mz + FLT(1.3425);
            hs.rho = FLT(-0.0165406) * Mz * Mz * Mz + FLT(0.2290201) * Mz * Mz - FLT(1.1069031) * Mz + FLT(3.0455);
        } else {
            vr = FLT(-0.0024324) * Mz + FLT(1.0019);
            hs.rho = FLT(-0.0012973) * Mz + FLT(1.1565);
        }
        if(Mz >= FLT(-1.0) && Mz < FLT(0.0)) alpha2_f = FLT(0.4556);
        else if(Mz >= FLT(0.0) && Mz < FLT(2.6)) alpha2_f = FLT(0.4556) + FLT(0.0245) * Mz;
        else if(Mz >= FLT(2.6) && Mz < FLT(4.5)) alpha2_f = FLT(0.1978) + FLT(0.1245) * Mz;
        else if(Mz >= FLT(4.5) && Mz < FLT(6.0)) alpha2_f = FLT(8.0399) - FLT(2.5228) * Mz + FLT(0.20098) * Mz * Mz;
        else if(Mz >= FLT(6.0) && Mz < FLT(9.5)) alpha2_f = FLT(0.9431) - FLT(0.2041) * Mz + FLT(0.0117) * Mz * Mz;
        else alpha2_f = FLT(0.0601);
        double alphaR = vr * FLT(1500.0);
        double alphaI = alpha2_f * (vr / FLT(1000.0)) * FLT(1500.0) * log(FLT(10.0)) / (FLT(40.0) * PI);
        const char L[2] = {'L', ' '};
        hs.cP = crci(env, fT, h[0], alphaR, alphaI, L);
        hs.cS = 0.0;
    }
    return hs;
}

/* src/curves.hpp:76-188 (de Boor cubic spline, complex ordinates) */
static void cspline(const double *tau, cpx *c1, cpx *c2, cpx *c3, cpx *c4, int n, int ibcbeg, int ibcend)
{
    cpx g = 0, dtau, divdf1, divdf3;
    int l = n - 1;
    for(int m = 1; m < n; ++m) {
        c3[m] = CMPLX(tau[m] - tau[m - 1], FLT(0.0));
        c4[m] = (c1[m] - c1[m - 1]) / c3[m];
    }
    if(ibcbeg == 0) {
        if(n > 2) {
            c4[0] = c3[2];
            c3[0] = c3[1] + c3[2];
            c2[0] = ((c3[1] + FLT(2.0) * c3[0]) * c4[1] * c3[2] + (c3[1] * c3[1]) * c4[2]) / c3[0];
        } else {
            c4[0] = CMPLX(1.0, 0.0);
            c3[0] = CMPLX(1.0, 0.0);
            c2[0] = FLT(2.0) * c4[1];
        }
    } else if(ibcbeg == 1) {
        c4[0] = CMPLX(1.0, 0.0);
        c3[0] = CMPLX(0.0, 0.0);
    } else if(ibcbeg == 2) {
        c4[0] = CMPLX(2.0, 0.0);
        c3[0] = CMPLX(1.0, 0.0);
        c2[0] = FLT(3.0) * c4[1] - c2[0] * c3[1] * FLT(0.5);
    }
    for(int m = 1; m < l; ++m) {
        g = -c3[m + 1] / c4[m - 1];
        c2[m] = g * c2[m - 1] + FLT(3.0) * (c3[m] * c4[m + 1] + c3[m + 1] * c4[m]);
        c4[m] = g * c3[m - 1] + FLT(2.0) * (c3[m] + c3[m + 1]);
    }
    if(ibcend != 1) {
        if(ibcend == 0) {
            if(n == 2 && ibcbeg == 0) {
                c2[n - 1] = c4[n - 1];
            } else if((n == 3 && ibcbeg == 0) || n == 2) {
                c2[n - 1] = FLT(2.0) * c4[n - 1];
                c4[n - 1] = CMPLX(1.0, 0.0);
                g = FLT(1.0) / -c4[n - 2];
            } else {
                g = c3[n - 2] + c3[n - 1];
                c2[n - 1] = ((c3[n - 1] + FLT(2.0) * g) * c4[n - 1] * c3[n - 2]
                             + (c3[n - 1] * c3[n - 1]) * (c1[n - 2] - c1[n - 3]) / c3[n - 2]) / g;
                g = -g / c4[n - 2];
                c4[n - 1] = c3[n - 2];
            }
        } else if(ibcend == 2) {
            c2[n - 1] = FLT(3.0) * c4[n - 1] + c2[n - 1] * c3[n - 1] * FLT(0.5);
            c4[n - 1] = CMPLX(2.0, 0.0);
            g = FLT(1.0) / -c4[n - 2];
        }
        if(ibcbeg > 0 || n > 2) {
            c4[n - 1] += g * c3[n - 2];
            c2[n - 1] = (g * c2[n - 2] + c2[n - 1]) / c4[n - 1];
        }
    }
    for(int j = l - 1; j >= 0; --j) c2[j] = (c2[j] - c3[j] * c2[j + 1]) / c4[j];
    for(int i = 1; i < n; ++i) {
        dtau = c3[i];
        divdf1 = (c1[i] - c1[i - 1]) / dtau;
        divdf3 = c2[i - 1] + c2[i] - FLT(2.0) * divdf1;
        c3[i - 1] = FLT(2.0) * (divdf1 - c2[i - 1] - divdf3) / dtau;
        c4[i - 1] = (divdf3 / dtau) * (FLT(6.0) / dtau);
    }
    c3[n - 1] = c3[l - 1] + (tau[n - 1] - tau[l - 1]) * c4[l - 1];
    c4[n - 1] = CMPLX(0.0, 0.0);
    for(int i = 0; i < l; ++i) {
        double dt = tau[i + 1] - tau[i];
        c4[n - 1] += dt * (c1[i] + dt * (c2[i] * FLT(0.5) + dt * (c3[i] / FLT(6.0) + dt * c4[i] / FLT(24.0))));
    }
    c4[n - 1] /= tau[n - 1] - tau[0];
}

/* src/curves.hpp:213-262 (monotone derivative projections) */
static double fp_interior(double d1, double d2, double fp)
{
    if(d1 * d2 > FLT(0.0)) {
        if(d1 > FLT(0.0)) return dmin(dmax(fp, 0.0), 3.0 * dmin(d1, d2));
        return dmax(dmin(fp, 0.0), 3.0 * dmax(d1, d2));
    }
    return 0.0;
}
static double fp_left(double d1, double d2, double fp)
{
    if(d1 * fp <= 0.0) return FLT(0.0);
    if((d1 * d2 <= 0.0) && (fabs(fp) > fabs(3.0 * d1))) return 3.0 * d1;
    return fp;
}

/* src/curves.hpp:299-372 (PCHIP) */
static void pchip(const double *x, const cpx *y, int n, cpx *pc1, cpx *pc2, cpx *pc3, cpx *pc4,
                  cpx *w1, cpx *w2, cpx *w3, cpx *w4)
{
    if(n == 2) {
        pc1[0] = y[0];
        pc2[0] = (y[1] - y[0]) / (x[1] - x[0]);
        pc3[0] = 0.0;
        pc4[0] = 0.0;
        return;
    }
    for(int i = 0; i < n; ++i) pc1[i] = y[i];
    double h1, h2;
    cpx del1, del2, ft;
    /* h_del src/curves.hpp:206-211 */
#define HDEL(ix) do { h1 = x[ix] - x[(ix) - 1]; h2 = x[(ix) + 1] - x[ix]; \
        del1 = (y[ix] - y[(ix) - 1]) / h1; del2 = (y[(ix) + 1] - y[ix]) / h2; } while(0)
    HDEL(1);
    ft = ((2.0 * h1 + h2) * del1 - h1 * del2) / (h1 + h2);
    pc2[0] = CMPLX(fp_left(creal(del1), creal(del2), creal(ft)), fp_left(cimag(del1), cimag(del2), cimag(ft)));
    HDEL(n - 2);
    ft = (-h2 * del1 + (h1 + 2.0 * h2) * del2) / (h1 + h2);
    pc2[n - 1] = CMPLX(fp_left(creal(del2), creal(del1), creal(ft)), fp_left(cimag(del2), cimag(del1), cimag(ft)));
    for(int i = 0; i < n; ++i) w1[i] = pc1[i];
    w2[0] = pc2[0];
    w2[n - 1] = pc2[n - 1];
    cspline(x, w1, w2, w3, w4, n, 1, 1);
    for(int ix = 1; ix < n - 1; ++ix) {
        HDEL(ix);
        pc2[ix] = CMPLX(fp_interior(creal(del1), creal(del2), creal(w2[ix])),
                        fp_interior(cimag(del1), cimag(del2), cimag(w2[ix])));
    }
#undef HDEL
    for(int ix = 0; ix < n - 1; ++ix) {
        double h = x[ix + 1] - x[ix];
        cpx f1 = pc1[ix], f2 = pc1[ix + 1], f1p = pc2[ix], f2p = pc2[ix + 1];
        pc3[ix] = (3.0 * (f2 - f1) - h * (2.0 * f1p + f2p)) / (h * h);
        pc4[ix] = (h * (f1p + f2p) - 2.0 * (f2 - f1)) / (h * h * h);
    }
}

/* src/common_setup.hpp:306-334 (SubTab, double and float) */
static void subtab_d(double *x, int n)
{
    if(n >= 3 && fabs(x[2] - (-999.9)) < 0.01) {
        if(fabs(x[1] - (-999.9)) < 0.01) x[1] = x[0];
        double dx = (x[1] - x[0]) / (double)(n - 1), x0 = x[0];
        for(int i = 0; i < n; ++i) x[i] = fma((double)i, dx, x0);
    }
}
static void subtab_f(float *x, int n)
{
    if(n >= 3 && fabsf(x[2] - (-999.9f)) < 0.01f) {
        if(fabsf(x[1] - (-999.9f)) < 0.01f) x[1] = x[0];
        float dx = (x[1] - x[0]) / (float)(n - 1), x0 = x[0];
        for(int i = 0; i < n; ++i) x[i] = fmaf((float)i, dx, x0);
    }
}
static int cmp_d(const void *a, const void *b)
{
    double x = *(const double *)a, y = *(const double *)b;
    return (x < y) ? -1 : (x > y);
}
static int cmp_f(const void *a, const void *b)
{
    float x = *(const float *)a, y = *(const float *)b;
    return (x < y) ? -1 : (x > y);
}

/* src/module/boundary.hpp:600-896 (2-D branch of ComputeBdryTangentNormal) */
static void bdry_tangent_normal(Bdry *b, double negtop)
{
    int n = b->n;
    for(int i = 0; i < n - 1; ++i) {
        BdPt *p = &b->bd[i];
        p->t = vsub(b->bd[i + 1].x, p->x);
        p->Dx = p->t.y / p->t.x;
        p->Len = vlen(p->t);
        p->t = vdiv(p->t, p->Len);
        p->n.x = -negtop * p->t.y;
        p->n.y = negtop * p->t.x;
    }
    if(b->type[0] == 'C') {
        for(int i = 1; i < n - 1; ++i) {
            double sss = FLT(0.5);
            b->bd[i].Nodet = vadd(vsc(FLT(1.0) - sss, b->bd[i - 1].t), vsc(sss, b->bd[i].t));
        }
        b->bd[0].Nodet = V(1.0, 0.0);
        b->bd[n - 1].Nodet = V(1.0, 0.0);
        for(int i = 0; i < n; ++i) {
            b->bd[i].Noden.x = -negtop * b->bd[i].Nodet.y;
            b->bd[i].Noden.y = negtop * b->bd[i].Nodet.x;
        }
        double curphi = atan2(b->bd[0].Nodet.y, b->bd[0].Nodet.x);
        for(int i = 0; i < n - 1; ++i) {
            double nextphi = atan2(b->bd[i + 1].Nodet.y, b->bd[i + 1].Nodet.x);
            b->bd[i].kappa = (nextphi - curphi) / b->bd[i].Len;
            b->bd[i].Dxx = (b->bd[i + 1].Dx - b->bd[i].Dx) / (b->bd[i + 1].x.x - b->bd[i].x.x);
            b->bd[i].Dss = b->bd[i].Dxx * b->bd[i].t.x * b->bd[i].t.x * b->bd[i].t.x;
            b->bd[i].kappa = b->bd[i].Dss;
            curphi = nextphi;
        }
    } else {
        for(int i = 0; i < n; ++i) b->bd[i].kappa = FLT(0.0);
    }
}

/* src/module/boundary.hpp:51-67,180-228,499-545 */
static void build_bdry(const O2Env *env, Bdry *b, int istop)
{
    double big = sqrt(DBL_MAX) / 1.0e5; /* src/boundary.hpp:26-34 */
    double depth = istop ? env->ssp_z[0] : env->bot_depth;
    char flag = istop ? env->top_file : env->bot_file;
    int has_file = (flag == '~' || flag == '*');
    if(!has_file) {
        b->n = 2;
        b->type[0] = 'L'; b->type[1] = 'S';
        b->bd = calloc(2, sizeof(BdPt));
        b->bd[0].x = V(-big, depth);
        b->bd[1].x = V(big, depth);
    } else {
        int np = istop ? env->ntop : env->nbot;
        const double *r = istop ? env->top_r : env->bot_r;
        const double *z = istop ? env->top_z : env->bot_z;
        const double *geo = istop ? env->top_geo : env->bot_geo;
        memcpy(b->type, istop ? env->top_type : env->bot_type, 2);
        b->n = np + 2;
        b->bd = calloc(b->n, sizeof(BdPt));
        for(int i = 1; i < b->n - 1; ++i) {
            b->bd[i].x = V(r[i - 1], z[i - 1]);
            if(b->type[1] == 'L') {
                const double *g = geo + 5 * (i - 1);
                const char W[2] = {'W', ' '};
                b->bd[i].hs.cP = crci(env, 0, 1.0e20, g[0], g[3], W);
                b->bd[i].hs.cS = crci(env, 0, 1.0e20, g[1], g[4], W);
                b->bd[i].hs.rho = g[2];
            }
        }
        b->bd[0].x = V(-big * 0.001, b->bd[1].x.y);
        b->bd[0].hs = b->bd[1].hs;
        b->bd[b->n - 1].x = V(big * 0.001, b->bd[b->n - 2].x.y);
        b->bd[b->n - 1].hs = b->bd[b->n - 2].hs;
    }
    for(int i = 0; i < b->n; ++i) b->bd[i].x.x *= 1000.0; /* km -> m */
    bdry_tangent_normal(b, istop ? -1.0 : 1.0);
}

static int build_env(const O2Env *in, Env *e, O2Out *out)
{
    memset(e, 0, sizeof(*e));
    memcpy(e->run_type, in->run_type, 7);
    /* module/runtype.hpp:63-78 normalisation */
    switch(e->run_type[1]) {
    case 'C': case 'R': case 'S': case 'b': case 'B': case 'g': break;
    default: e->run_type[1] = 'G';
    }
    if(e->run_type[3] != 'X') e->run_type[3] = 'R';
    if(e->run_type[4] != 'I') e->run_type[4] = 'R';
    /* module/beaminfo.hpp:240-244 MoveBeamType */
    memcpy(e->beam_type, "G S ", 4);
    e->beam_type[0] = e->run_type[1];
    e->beam_type[3] = e->run_type[6];
    e->freq0 = in->freq0;
    e->type = in->ssp_type;
    /* fT: 1e20 from BoundaryCond::SetupPre, 1000 after reading an 'A' bottom
       (module/boundarycond.hpp:37-58; modules run SetupPre/Read in order, api.cpp:271-276) */
    double fT = (in->bot_bc == 'A') ? FLT(1000.0) : 1.0e20;

    /* SSP (module/ssp.hpp:453-545) */
    int n = in->nssp;
    e->npts = n;
    e->z = calloc(n, sizeof(double));
    e->rho = calloc(n, sizeof(double));
    e->c = calloc(n, sizeof(cpx));
    e->cz = calloc(n, sizeof(cpx));
    e->n2 = calloc(n, sizeof(cpx));
    e->n2z = calloc(n, sizeof(cpx));
    for(int k = 0; k < 4; ++k) {
        e->spl[k] = calloc(n, sizeof(cpx));
        e->coef[k] = calloc(n, sizeof(cpx));
    }
    for(int i = 0; i < n; ++i) {
        e->z[i] = in->ssp_z[i];
        e->rho[i] = in->ssp_rho[i];
        e->c[i] = crci(in, fT, in->ssp_z[i], in->ssp_alphaR[i], in->ssp_alphaI[i], in->atten_unit);
        if(i > 0) e->cz[i - 1] = (e->c[i] - e->c[i - 1]) / (e->z[i] - e->z[i - 1]);
    }
    e->cz[n - 1] = CMPLX(NAN, NAN);
    if(e->type == 'N') {
        for(int i = 0; i < n; ++i) e->n2[i] = FLT(1.0) / (e->c[i] * e->c[i]);
        for(int i = 1; i < n; ++i) e->n2z[i - 1] = (e->n2[i] - e->n2[i - 1]) / (e->z[i] - e->z[i - 1]);
    } else if(e->type == 'S') {
        for(int i = 0; i < n; ++i) e->spl[0][i] = e->c[i];
        cspline(e->z, e->spl[0], e->spl[1], e->spl[2], e->spl[3], n, 0, 0);
    } else if(e->type == 'P') {
        cpx *w[4];
        for(int k = 0; k < 4; ++k) w[k] = calloc(n, sizeof(cpx));
        pchip(e->z, e->c, n, e->coef[0], e->coef[1], e->coef[2], e->coef[3], w[0], w[1], w[2], w[3]);
        for(int k = 0; k < 4; ++k) free(w[k]);
    } else if(e->type != 'C' && e->type != 'A') {
        return -1;
    }
    e->top_depth = in->ssp_z[0];
    e->bot_depth = in->bot_depth;
    e->top = make_hs(in, fT, in->top_bc, in->top_hs);
    e->bot = make_hs(in, fT, in->bot_bc, in->bot_hs);
    build_bdry(in, &e->btop, 1);
    build_bdry(in, &e->bbot, 0);

    /* source / receiver depths (module/szrz.hpp:64-125) */
    e->nsz = in->nsz;
    e->sz = calloc(imax(3, in->nsz), sizeof(float));
    memcpy(e->sz, in->sz_in, imax(3, in->nsz) * sizeof(float));
    subtab_f(e->sz, e->nsz);
    qsort(e->sz, e->nsz, sizeof(float), cmp_f);
    e->nrz = in->nrz;
    e->rz = calloc(imax(3, in->nrz), sizeof(float));
    memcpy(e->rz, in->rz_in, imax(3, in->nrz) * sizeof(float));
    subtab_f(e->rz, e->nrz);
    qsort(e->rz, e->nrz, sizeof(float), cmp_f);
    for(int i = 0; i < e->nsz; ++i) {
        if(e->sz[i] < e->top_depth) e->sz[i] = (float)e->top_depth;
        if(e->sz[i] > e->bot_depth) e->sz[i] = (float)e->bot_depth;
    }
    for(int i = 0; i < e->nrz; ++i) {
        if(e->rz[i] < e->top_depth) e->rz[i] = (float)e->top_depth;
        if(e->rz[i] > e->bot_depth) e->rz[i] = (float)e->bot_depth;
    }
    /* receiver ranges (module/rcvrranges.hpp:80-85) */
    e->nrr = in->nrr;
    e->rr = calloc(imax(3, in->nrr), sizeof(double));
    memcpy(e->rr, in->rr_in, imax(3, in->nrr) * sizeof(double));
    subtab_d(e->rr, e->nrr);
    qsort(e->rr, e->nrr, sizeof(double), cmp_d);
    for(int i = 0; i < e->nrr; ++i) e->rr[i] *= FLT(1000.0);
    e->delta_r = (e->nrr >= 2) ? e->rr[e->nrr - 1] - e->rr[e->nrr - 2] : FLT(0.0);
    e->nrz_per_range = (e->run_type[4] == 'I') ? 1 : e->nrz;

    /* angles (module/rayangles.hpp:66-190) */
    int na = in->nalpha;
    if(na == 0) {
        double c0 = FLT(1500.0);
        na = imax((int)(FLT(0.3) * e->rr[e->nrr - 1] * e->freq0 / c0), 300);
        double depth = e->bot_depth - e->top_depth;
        double dth = atan(depth / (FLT(10.0) * e->rr[e->nrr - 1]));
        na = imax((int)(PI / dth), na);
    }
    e->nalpha = na;
    e->alpha = calloc(imax(3, na), sizeof(double));
    if(in->nalpha > 0) {
        memcpy(e->alpha, in->alpha_in, imax(3, na) * sizeof(double));
    } else {
        e->alpha[0] = in->alpha_in[0];
        e->alpha[1] = in->alpha_in[1];
        e->alpha[2] = -999.9;
    }
    if(na > 2 && in->nalpha == 0) e->alpha[2] = FLT(-999.9);
    subtab_d(e->alpha, na);
    qsort(e->alpha, na, sizeof(double), cmp_d);
    if(na > 1 && fabs(fmod(e->alpha[na - 1] - e->alpha[0], FLT(360.0))) < FLT(10.0) * spacing(360.0))
        --na; /* src/common_setup.hpp:257-270 */
    e->nalpha = na;
    for(int i = 0; i < na; ++i) e->alpha[i] *= DEG_RAD;
    e->dalpha = (na != 1) ? (e->alpha[na - 1] - e->alpha[0]) / (na - 1) : FLT(0.0);
    e->isingle = in->isingle;

    /* beam (module/beaminfo.hpp:220-237) */
    e->box_x = in->box_r_km * FLT(1000.0);
    e->box_y = in->box_z;
    e->deltas = in->deltas;
    if(fabs(e->deltas) < REAL_EPS) e->deltas = (e->bot_depth - e->top_depth) / FLT(10.0);

    /* source beam pattern (module/sbp.hpp:58-67,148-157) */
    if(in->nsbp > 0) {
        e->nsbp = in->nsbp;
        e->sbp = calloc(2 * in->nsbp, sizeof(double));
        for(int i = 0; i < in->nsbp; ++i) {
            e->sbp[2 * i] = in->sbp[2 * i];
            e->sbp[2 * i + 1] = pow(FLT(10.0), in->sbp[2 * i + 1] / FLT(20.0));
        }
    } else {
        e->nsbp = 2;
        e->sbp = calloc(4, sizeof(double));
        e->sbp[0] = FLT(-180.0); e->sbp[1] = pow(FLT(10.0), 0.0 / FLT(20.0));
        e->sbp[2] = FLT(180.0); e->sbp[3] = pow(FLT(10.0), 0.0 / FLT(20.0));
    }
    e->max_narr = in->max_narr;
    e->allow_merging = in->allow_merging;
    e->eigen_memsize = in->eigen_memsize;
    if(out) {
        out->NSz = e->nsz;
        out->NRz = e->nrz;
        out->NRz_per_range = e->nrz_per_range;
        out->NRr = e->nrr;
        out->Nalpha = (e->isingle > 0) ? 1 : e->nalpha;
    }
    return 0;
}

static void free_env(Env *e)
{
    free(e->z); free(e->rho); free(e->c); free(e->cz); free(e->n2); free(e->n2z);
    for(int k = 0; k < 4; ++k) { free(e->spl[k]); free(e->coef[k]); }
    free(e->btop.bd); free(e->bbot.bd);
    free(e->sz); free(e->rz); free(e->rr); free(e->alpha); free(e->sbp);
}

/* ------------------------------------------------------------------ */
/* run-time: SSP evaluation (src/ssp.hpp)                               */
/* ------------------------------------------------------------------ */
typedef struct { v2 gradc; cpx ccpx; double rho, czz, crr, crz; } SSPOut;
typedef struct { int r, z; } SegSt;

/* src/ssp.hpp:36-51 */
static void update_seg(double x, double t, const double *a, int n, int *iSeg)
{
    if(t >= 0.0) {
        while(*iSeg > 0 && x < a[*iSeg]) --*iSeg;
        while(*iSeg < n - 2 && x >= a[*iSeg + 1]) ++*iSeg;
    } else {
        while(*iSeg < n - 2 && x > a[*iSeg + 1]) ++*iSeg;
        while(*iSeg > 0 && x <= a[*iSeg]) --*iSeg;
    }
}
/* src/ssp.hpp:53-59 */
static double lin_rho(double z, const Env *e, int iz, double *rho)
{
    double w = (z - e->z[iz]) / (e->z[iz + 1] - e->z[iz]);
    *rho = (1.0 - w) * e->rho[iz] + w * e->rho[iz + 1];
    return w;
}

/* src/ssp.hpp:64-152,309-375,377-465 (2-D, 1-D profile types) */
static void eval_ssp(v2 x, v2 t, SSPOut *o, const Env *e, SegSt *s, ErrSt *err)
{
    o->crr = o->crz = o->czz = 0.0;
    switch(e->type) {
    case 'N': {
        update_seg(x.y, t.y, e->z, e->npts, &s->z);
        double w = lin_rho(x.y, e, s->z, &o->rho);
        o->ccpx = 1.0 / csqrt((1.0 - w) * e->n2[s->z] + w * e->n2[s->z + 1]);
        double c = creal(o->ccpx);
        o->gradc = V(0.0, -0.5 * (c * c * c) * creal(e->n2z[s->z]));
        o->czz = 3.0 * o->gradc.y * o->gradc.y / c;
    } break;
    case 'C':
        update_seg(x.y, t.y, e->z, e->npts, &s->z);
        lin_rho(x.y, e, s->z, &o->rho);
        o->ccpx = e->c[s->z] + (x.y - e->z[s->z]) * e->cz[s->z];
        o->gradc = V(0.0, creal(e->cz[s->z]));
        break;
    case 'S': {
        update_seg(x.y, t.y, e->z, e->npts, &s->z);
        lin_rho(x.y, e, s->z, &o->rho);
        double h = x.y - e->z[s->z];
        int i = s->z;
        const double half = FLT(0.5), sixth = (double)(1.0f / 6.0f);
        /* SplineALL src/curves.hpp:190-204 */
        o->ccpx = e->spl[0][i] + h * (e->spl[1][i] + h * (half * e->spl[2][i] + sixth * h * e->spl[3][i]));
        cpx fx = e->spl[1][i] + h * (e->spl[2][i] + h * half * e->spl[3][i]);
        cpx fxx = e->spl[2][i] + h * e->spl[3][i];
        o->gradc = V(0.0, creal(fx));
        o->czz = creal(fxx);
    } break;
    case 'P': {
        update_seg(x.y, t.y, e->z, e->npts, &s->z);
        lin_rho(x.y, e, s->z, &o->rho);
        int i = s->z;
        double xt = x.y - e->z[i];
        if(fabs(xt) > 1.0e10) run_warn(err, W_PCHIP_XT);
        for(int k = 0; k < 4; ++k)
            if(cabs(e->coef[k][i]) > 1.0e10) run_warn(err, W_PCHIP_COEF);
        o->ccpx = e->coef[0][i] + (e->coef[1][i] + (e->coef[2][i] + e->coef[3][i] * xt) * xt) * xt;
        o->gradc = V(0.0, creal(e->coef[1][i] + (2.0 * e->coef[2][i] + 3.0 * e->coef[3][i] * xt) * xt));
        o->czz = creal(2.0 * e->coef[2][i] + 6.0 * e->coef[3][i] * xt);
    } break;
    case 'A': {
        s->z = 0;
        double c0 = FLT(1500.0);
        o->rho = FLT(1.0);
        const double u1 = FLT(1300.0), u2 = FLT(0.00737);
        double xt = FLT(2.0) * (x.y - u1) / u1;
        double emxt = exp(-xt);
        double dxt = FLT(2.0) / u1;
        o->ccpx = CMPLX(c0 * (FLT(1.0) + u2 * (xt - FLT(1.0) + emxt)), FLT(0.0));
        double cz = c0 * u2 * (FLT(1.0) - emxt) * dxt;
        o->czz = c0 * u2 * emxt * dxt * dxt;
        o->gradc = V(FLT(0.0), cz);
    } break;
    default: run_error(err, E_SSP_TYPE);
    }
}

/* ------------------------------------------------------------------ */
/* boundaries, step (src/boundary.hpp, src/step.hpp, src/trace.hpp)      */
/* ------------------------------------------------------------------ */
typedef struct { int Iseg; double lmin, lmax; v2 x, n; } BdSt;
typedef struct {
    int NumTopBnc, NumBotBnc;
    v2 x, t, p, q;
    double c, Amp, Phase;
    cpx tau;
} RayPt; /* include/bhc/structs.hpp:397-424 (2-D) */

/* src/boundary.hpp:66-227 (2-D branch) */
static void get_bdry_seg(v2 x, v2 t, BdSt *bs, const Bdry *b, HS *hs, int istop, int isinit, ErrSt *err)
{
    if(!isinit && !(x.x < bs->lmin || (x.x == bs->lmin && t.x < 0.0) || x.x > bs->lmax
                    || (x.x == bs->lmax && t.x >= 0.0)))
        return;
    int n = b->n;
    bs->Iseg = imin(imax(bs->Iseg, 0), n - 2);
    if(t.x >= 0.0) {
        while(bs->Iseg >= 0 && b->bd[bs->Iseg].x.x > x.x) --bs->Iseg;
        while(bs->Iseg >= 0 && bs->Iseg < n - 1 && b->bd[bs->Iseg + 1].x.x <= x.x) ++bs->Iseg;
    } else {
        while(bs->Iseg < n - 1 && b->bd[bs->Iseg + 1].x.x < x.x) ++bs->Iseg;
        while(bs->Iseg >= 0 && bs->Iseg < n - 1 && b->bd[bs->Iseg].x.x >= x.x) --bs->Iseg;
    }
    if(bs->Iseg < 0 || bs->Iseg >= n - 1) {
        run_error(err, istop ? E_OUT_ALT : E_OUT_BTY);
        bs->Iseg = 0;
    }
    bs->lmin = b->bd[bs->Iseg].x.x;
    bs->lmax = b->bd[bs->Iseg + 1].x.x;
    bs->x = b->bd[bs->Iseg].x;
    bs->n = b->bd[bs->Iseg].n;
    if(b->type[1] == 'L') {
        hs->cP = b->bd[bs->Iseg].hs.cP;
        hs->cS = b->bd[bs->Iseg].hs.cS;
        hs->rho = b->bd[bs->Iseg].hs.rho;
    }
}

/* src/trace.hpp:37-45 */
static void distances(v2 x, const BdSt *top, const BdSt *bot, double *dt, double *db)
{
    *dt = -vdot(top->n, vsub(x, top->x));
    *db = -vdot(bot->n, vsub(x, bot->x));
}

static inline double dim_of(v2 v, int d) { return d == 0 ? v.x : v.y; }
static inline void set_dim(v2 *v, int d, double s) { if(d == 0) v->x = s; else v->y = s; }

/* src/common_run.hpp:49-53 (box centred on (0,0) in 2-D) */
static int outside_box(v2 x, const Env *e, int d)
{
    return fabs(dim_of(x, d) - 0.0) >= (d == 0 ? e->box_x : e->box_y);
}

/* src/step.hpp:41-79 */
static void depth_iface(int stepTo, double *h, v2 *x, v2 x0, v2 u, SegSt s0, const Env *e)
{
    if(!stepTo) *h = DBL_MAX;
    if(fabs(u.y) > REAL_EPS) {
        if(e->z[s0.z] > x->y) {
            *h = (e->z[s0.z] - x0.y) / u.y;
            if(stepTo) { *x = vadd(x0, vsc(*h, u)); x->y = e->z[s0.z]; }
        } else if(e->z[s0.z + 1] < x->y) {
            *h = (e->z[s0.z + 1] - x0.y) / u.y;
            if(stepTo) { *x = vadd(x0, vsc(*h, u)); x->y = e->z[s0.z + 1]; }
        }
    }
}
/* src/step.hpp:84-108 */
static void box_cross(int stepTo, int d, double *h, v2 *x, v2 x0, v2 u, const Env *e)
{
    if(!stepTo) *h = DBL_MAX;
    if(outside_box(*x, e, d)) {
        double box = d == 0 ? e->box_x : e->box_y;
        double d0 = dim_of(x0, d) - 0.0;
        *h = (box - fabs(d0)) / fabs(dim_of(u, d));
        if(stepTo) { *x = vadd(x0, vsc(*h, u)); set_dim(x, d, 0.0 + copysign(box, d0)); }
    }
}
/* src/step.hpp:113-147 */
static void topbot_cross(int stepTo, double *h, const BdSt *bd, v2 *x, v2 x0, v2 u, int *refl)
{
    if(!stepTo) *h = DBL_MAX;
    v2 d = vsub(*x, bd->x), d0 = vsub(x0, bd->x);
    double w = vdot(bd->n, d);
    if(stepTo ? (w > -INF_STEP) : (w >= 0.0)) {
        *h = -vdot(d0, bd->n) / vdot(u, bd->n);
        if(stepTo) {
            *x = vadd(x0, vsc(*h, u));
            if(fabs(bd->n.x) < REAL_EPS) x->y = bd->x.y;
        }
        *refl = 1;
    } else {
        *refl = 0;
    }
}
/* src/step.hpp:153-205 (range branch) */
static void seg_cross(int stepTo, double *h, const BdSt *top, const BdSt *bot, v2 *x, v2 x0, v2 u,
                      int *trefl, int *brefl)
{
    double lmin = dmax(top->lmin, bot->lmin), lmax = dmin(top->lmax, bot->lmax);
    if(!stepTo) *h = DBL_MAX;
    if(fabs(u.x) > REAL_EPS) {
        if(x->x < lmin) {
            *h = -(x0.x - lmin) / u.x;
            if(stepTo) { *x = vadd(x0, vsc(*h, u)); x->x = lmin; *trefl = *brefl = 0; }
        } else if(x->x > lmax) {
            *h = -(x0.x - lmax) / u.x;
            if(stepTo) { *x = vadd(x0, vsc(*h, u)); x->x = lmax; *trefl = *brefl = 0; }
        }
    }
}
/* src/step.hpp:271-342 */
static void reduce_step(v2 x0, v2 u, SegSt s0, BdSt *top, BdSt *bot, const Env *e, ErrSt *err,
                        double *h, int *small)
{
    double hInt, hB0, hB1, hTop, hBot, hSeg;
    int dummy;
    v2 x = vadd(x0, vsc(*h, u));
    depth_iface(0, &hInt, &x, x0, u, s0, e);
    box_cross(0, 0, &hB0, &x, x0, u, e);
    box_cross(0, 1, &hB1, &x, x0, u, e);
    double hBz = DBL_MAX;
    topbot_cross(0, &hTop, top, &x, x0, u, &dummy);
    topbot_cross(0, &hBot, bot, &x, x0, u, &dummy);
    seg_cross(0, &hSeg, top, bot, &x, x0, u, &dummy, &dummy);
    double hy = DBL_MAX, htd = DBL_MAX, hbd = DBL_MAX;
    *h = dmin(dmin(dmin(*h, hInt), dmin(dmin(dmin(hB0, hB1), hBz), dmin(hTop, hBot))),
              dmin(dmin(hSeg, hy), dmin(htd, hbd)));
    if(*h < -1e-4) run_warn(err, W_STEP_NEG);
    if(*h < INF_STEP * e->deltas) {
        *h = INF_STEP * e->deltas;
        ++*small;
    } else {
        *small = 0;
    }
}
/* src/step.hpp:347-424 */
static void step_to_bdry(v2 x0, v2 *x2, v2 u, double *h, int *trefl, int *brefl, SegSt s0,
                         BdSt *top, BdSt *bot, const Env *e)
{
    *x2 = vadd(x0, vsc(*h, u));
    depth_iface(1, h, x2, x0, u, s0, e);
    box_cross(1, 0, h, x2, x0, u, e);
    box_cross(1, 1, h, x2, x0, u, e);
    topbot_cross(1, h, top, x2, x0, u, trefl);
    topbot_cross(1, h, bot, x2, x0, u, brefl);
    if(*brefl) *trefl = 0;
    seg_cross(1, h, top, bot, x2, x0, u, trefl, brefl);
    if(*h < INF_STEP * e->deltas) {
        *h = INF_STEP * e->deltas;
        *x2 = vadd(x0, vsc(*h, u));
        v2 d = vsub(*x2, top->x);
        if(vdot(top->n, d) > REAL_EPS) *trefl = 1; else *trefl = 0;
        d = vsub(*x2, bot->x);
        if(vdot(bot->n, d) > REAL_EPS) { *brefl = 1; *trefl = 0; } else *brefl = 0;
    }
}

/* src/step.hpp:589-649 (2-D branch) */
static void curvature_correction(RayPt *ray, v2 gjump, SegSt s, SegSt s0)
{
    v2 ray2n = V(-ray->t.y, ray->t.x);
    double cnjump = vdot(gjump, ray2n);
    double csjump = vdot(gjump, ray->t);
    double rm;
    if(s.z != s0.z) rm = ray->t.x / ray->t.y;
    else rm = -ray->t.y / ray->t.x;
    double rn = rm * (FLT(2.0) * cnjump - rm * csjump) / ray->c;
    ray->p = vsub(ray->p, vsc(rn, ray->q));
}

/* src/step.hpp:654-811 */
static void step2d(RayPt ray0, RayPt *ray2, BdSt *top, BdSt *bot, const Env *e, SegSt *iSeg,
                   ErrSt *err, int *small, int *trefl, int *brefl)
{
    SSPOut o0, o1, o2;
    RayPt ray1;
    eval_ssp(ray0.x, ray0.t, &o0, e, iSeg, err);
    double cnn0 = o0.crr * ray0.t.y * ray0.t.y - FLT(2.0) * o0.crz * ray0.t.x * ray0.t.y
        + o0.czz * ray0.t.x * ray0.t.x;
    v2 pq0p = vsc(-cnn0, ray0.q), pq0q = vsc(creal(o0.ccpx), ray0.p);
    SegSt s0 = *iSeg;
    double c0 = creal(o0.ccpx);
    double csq0 = c0 * c0;
    v2 u0 = vsc(c0, ray0.t);
    double h = e->deltas;
    reduce_step(ray0.x, u0, s0, top, bot, e, err, &h, small);
    double halfh = FLT(0.5) * h;
    ray1.x = vadd(ray0.x, vsc(halfh, u0));
    ray1.t = vsub(ray0.t, vdiv(vsc(halfh, o0.gradc), csq0));
    ray1.p = vadd(ray0.p, vsc(halfh, pq0p));
    ray1.q = vadd(ray0.q, vsc(halfh, pq0q));

    eval_ssp(ray1.x, ray1.t, &o1, e, iSeg, err);
    double cnn1 = o1.crr * ray1.t.y * ray1.t.y - FLT(2.0) * o1.crz * ray1.t.x * ray1.t.y
        + o1.czz * ray1.t.x * ray1.t.x;
    v2 pq1p = vsc(-cnn1, ray1.q), pq1q = vsc(creal(o1.ccpx), ray1.p);
    double c1 = creal(o1.ccpx);
    double csq1 = c1 * c1;
    v2 u1 = vsc(c1, ray1.t);
    reduce_step(ray0.x, u1, s0, top, bot, e, err, &h, small);
    double w1 = h / (2.0 * halfh);
    double w0 = 1.0 - w1;
    v2 u2 = vadd(vsc(w0, u0), vsc(w1, u1));
    v2 x2;
    step_to_bdry(ray0.x, &x2, u2, &h, trefl, brefl, s0, top, bot, e);
    ray2->x = x2;
    double hw0 = h * w0, hw1 = h * w1;
    ray2->t = vsub(vsub(ray0.t, vdiv(vsc(hw0, o0.gradc), csq0)), vdiv(vsc(hw1, o1.gradc), csq1));
    ray2->tau = ray0.tau + hw0 / o0.ccpx + hw1 / o1.ccpx;
    ray2->p = vadd(ray0.p, vsc(hw0, pq0p));
    ray2->q = vadd(ray0.q, vsc(hw0, pq0q));
    ray2->p = vadd(ray2->p, vsc(hw1, pq1p));
    ray2->q = vadd(ray2->q, vsc(hw1, pq1q));
    ray2->Amp = ray0.Amp;
    ray2->Phase = ray0.Phase;
    ray2->NumTopBnc = ray0.NumTopBnc;
    ray2->NumBotBnc = ray0.NumBotBnc;
    eval_ssp(ray2->x, ray2->t, &o2, e, iSeg, err);
    ray2->c = creal(o2.ccpx);
    if(iSeg->z != s0.z || iSeg->r != s0.r)
        curvature_correction(ray2, vsub(o2.gradc, o0.gradc), *iSeg, s0);
}

/* src/reflect.hpp:125-452 (2-D branch; 'R','V','A','G'; beam shift not restated) */
static void reflect2d(RayPt old, RayPt *np, const HS *hs, int istop, v2 tB, v2 nB, double kappa,
                      const Env *e, SegSt *iSeg, ErrSt *err)
{
    double Th = vdot(old.t, nB);
    double Tg = vdot(old.t, tB);
    np->NumTopBnc = old.NumTopBnc + istop;
    np->NumBotBnc = old.NumBotBnc + (1 - istop);
    np->x = old.x;
    np->t = vsub(old.t, vsc(FLT(2.0) * Th, nB));
    SSPOut o;
    eval_ssp(old.x, old.t, &o, e, iSeg, err);
    double c = creal(o.ccpx);
    np->c = c;
    np->tau = old.tau;
    v2 rayt = vsc(c, old.t);
    v2 rayn = V(-rayt.y, rayt.x);
    v2 rayt_t = vsc(c, np->t);
    v2 rayn_t = V(rayt_t.y, -rayt_t.x); /* -vec2(-y, x) */
    double rn = FLT(2.0) * kappa / (c * c) / Th;
    double cnjump = -vdot(o.gradc, vsub(rayn_t, rayn));
    double csjump = -vdot(o.gradc, vsub(rayt_t, rayt));
    if(istop) { cnjump = -cnjump; rn = -rn; }
    double rm = Tg / Th;
    rn += rm * (FLT(2.0) * cnjump - rm * csjump) / (c * c);
    if(e->beam_type[2] == 'D') rn *= FLT(2.0);
    else if(e->beam_type[2] == 'Z') rn = FLT(0.0);
    np->p = vadd(old.p, vsc(rn, old.q));
    np->q = old.q;
    if(hs->bc == 'R') {
        np->Amp = old.Amp;
        np->Phase = old.Phase;
    } else if(hs->bc == 'V') {
        np->Amp = old.Amp;
        np->Phase = old.Phase + PI;
    } else if(hs->bc == 'A' || hs->bc == 'G') {
        double omega = FLT(2.0) * PI * e->freq0;
        cpx kx = omega * Tg, kz = omega * Th;
        cpx kx2 = kx * kx;
        cpx f, g;
        if(creal(hs->cS) > FLT(0.0)) {
            cpx kzS2 = kx2 - (omega / hs->cS) * (omega / hs->cS);
            cpx kzP2 = kx2 - (omega / hs->cP) * (omega / hs->cP);
            cpx kzS = csqrt(kzS2), kzP = csqrt(kzP2);
            cpx mu = hs->rho * (hs->cS * hs->cS);
            cpx y2 = ((kzS2 + kx2) * (kzS2 + kx2) - 4.0 * kzS * kzP * kx2) * mu;
            cpx y4 = kzP * (kx2 - kzS2);
            f = (omega * omega) * y4;
            g = y2;
        } else {
            cpx kzP = csqrt(kx2 - (omega / hs->cP) * (omega / hs->cP));
            if(fabs(creal(kzP)) < REAL_EPS && cimag(kzP) < 0.0) kzP = -kzP;
            f = kzP;
            g = hs->rho;
        }
        const cpx J = CMPLX(0.0, 1.0);
        cpx Refl = -(o.rho * f - J * kz * g) / (o.rho * f + J * kz * g);
        if(cabs(Refl) < FLT(1.0e-5)) {
            np->Amp = FLT(0.0);
            np->Phase = old.Phase;
        } else {
            np->Amp = cabs(Refl) * old.Amp;
            np->Phase = old.Phase + atan2(cimag(Refl), creal(Refl));
        }
    } else {
        run_error(err, E_BC_TYPE);
        np->Amp = NAN;
        np->Phase = NAN;
    }
}

/* ------------------------------------------------------------------ */
/* influence (src/influence.hpp), arrivals, eigen hits                  */
/* ------------------------------------------------------------------ */
typedef struct {
    int isz, ialpha;
    double alpha, SrcDeclAngle;
    double c0, freq0, omega, RadMax, BeamWindow, Ratio1, rcp_q0;
    double phase, qOld;
    v2 x;
    int ir;
} Infl;

typedef struct {
    const Env *e;
    O2Out *out;
    int gauss, coherent, tl, arrivals, eigen, also_eigen;
} Ctx;

/* src/common_run.hpp:61-138 */
static int bsearch_leq(const double *a, int n, int stride, int off, double t)
{
    int lo = 0, hi = n;
    while(lo < hi) {
        int m = (lo + hi) / 2;
        if(a[m * stride + off] > t) hi = m;
        else if(m >= n - 1) return n - 1;
        else if(a[(m + 1) * stride + off] > t) return m;
        else lo = m + 1;
    }
    return lo;
}
static int bsearch_gt(const double *a, int n, double t)
{
    int lo = -1, hi = n - 1;
    while(lo < hi) {
        int m = (lo + hi + 1) / 2;
        if(a[m] <= t) lo = m;
        else if(m <= 0) return 0;
        else if(a[m - 1] <= t) return m;
        else hi = m - 1;
    }
    return hi;
}

/* src/eigenrays.hpp:24-40 */
static void record_hit(Ctx *cx, int ir, int iz, int is, const Infl *inf)
{
    int mi = cx->out->neigen++;
    if(mi >= cx->e->eigen_memsize || !cx->out->hits) return;
    O2Hit *h = &cx->out->hits[mi];
    h->is = is; h->iz = iz; h->ir = ir; h->itheta = 0;
    h->isx = 0; h->isy = 0; h->isz = inf->isz; h->ialpha = inf->ialpha; h->ibeta = 0;
}

/* src/arrivals.hpp:31-132 */
static void add_arr(Ctx *cx, int iz, int ir, double Amp, double omega, double Phase, cpx delay,
                    const Infl *inf, double RcvrDecl, int ntop, int nbot)
{
    const Env *e = cx->e;
    size_t base = ((size_t)inf->isz * e->nrz_per_range + iz) * e->nrr + ir;
    O2Arrival *ba = &cx->out->arr[base * e->max_narr];
    int32_t *bn = &cx->out->narr[base];
    float azim = NAN;
    if(e->allow_merging) {
        int Nt = *bn;
        const float PhaseTol = 0.05f;
        int second = Nt >= 1
            && omega * cabs(delay - CMPLX((double)ba[Nt - 1].delay_re, (double)ba[Nt - 1].delay_im)) < PhaseTol
            && fabs(ba[Nt - 1].Phase - Phase) < PhaseTol;
        if(!second) {
            int iArr;
            if(Nt >= e->max_narr) {
                iArr = -1;
                double weakest = Amp;
                for(Nt = 0; Nt < e->max_narr; ++Nt) {
                    if(ba[Nt].a < weakest) { weakest = ba[Nt].a; iArr = Nt; }
                }
                if(iArr < 0) return;
            } else {
                iArr = Nt;
                *bn = Nt + 1;
            }
            ba[iArr].a = (float)Amp;
            ba[iArr].Phase = (float)Phase;
            ba[iArr].delay_re = (float)creal(delay);
            ba[iArr].delay_im = (float)cimag(delay);
            ba[iArr].SrcDeclAngle = (float)inf->SrcDeclAngle;
            ba[iArr].SrcAzimAngle = azim;
            ba[iArr].RcvrDeclAngle = (float)RcvrDecl;
            ba[iArr].RcvrAzimAngle = azim;
            ba[iArr].NTopBnc = ntop;
            ba[iArr].NBotBnc = nbot;
        } else {
            float AmpTot = ba[Nt - 1].a + (float)Amp;
            float w1 = ba[Nt - 1].a / AmpTot, w2 = (float)Amp / AmpTot;
            ba[Nt - 1].delay_re = w1 * ba[Nt - 1].delay_re + w2 * (float)creal(delay);
            ba[Nt - 1].delay_im = w1 * ba[Nt - 1].delay_im + w2 * (float)cimag(delay);
            ba[Nt - 1].a = AmpTot;
            ba[Nt - 1].SrcDeclAngle = w1 * ba[Nt - 1].SrcDeclAngle + w2 * (float)inf->SrcDeclAngle;
            ba[Nt - 1].SrcAzimAngle = w1 * ba[Nt - 1].SrcAzimAngle + w2 * azim;
            ba[Nt - 1].RcvrDeclAngle = w1 * ba[Nt - 1].RcvrDeclAngle + w2 * (float)RcvrDecl;
            ba[Nt - 1].RcvrAzimAngle = w1 * ba[Nt - 1].RcvrAzimAngle + w2 * azim;
        }
    } else {
        int Nt = (*bn)++;
        if(Nt >= e->max_narr) return;
        ba[Nt].a = (float)Amp;
        ba[Nt].Phase = (float)Phase;
        ba[Nt].delay_re = (float)creal(delay);
        ba[Nt].delay_im = (float)cimag(delay);
        ba[Nt].SrcDeclAngle = (float)inf->SrcDeclAngle;
        ba[Nt].SrcAzimAngle = azim;
        ba[Nt].RcvrDeclAngle = (float)RcvrDecl;
        ba[Nt].RcvrAzimAngle = azim;
        ba[Nt].NTopBnc = ntop;
        ba[Nt].NBotBnc = nbot;
    }
}

/* src/influence.hpp:432-473 */
static void apply_contrib(Ctx *cx, double cnst, double w, double omega, cpx delay, double phaseInt,
                          double RcvrDecl, int ir, int iz, int is, const Infl *inf, const RayPt *p1)
{
    const Env *e = cx->e;
    cx->out->nevals++;
    if(cx->eigen) {
        record_hit(cx, ir, iz, is, inf);
    } else if(cx->arrivals) {
        if(cx->out->arr) add_arr(cx, iz, ir, cnst * w, omega, phaseInt, delay, inf, RcvrDecl, p1->NumTopBnc, p1->NumBotBnc);
        if(cx->also_eigen) record_hit(cx, ir, iz, is, inf);
    } else if(cx->out->field) {
        float re, im;
        if(cx->coherent) {
            const cpx J = CMPLX(0.0, 1.0);
            cpx z = omega * delay - phaseInt;
            cpx v = (cnst * w) * cexp(-J * z);
            re = (float)creal(v);
            im = (float)cimag(v);
        } else {
            double v = cnst * exp(cimag(omega * delay));
            v = v * v * w;
            if(cx->gauss) v *= sqrt(FLT(2.0) * PI);
            re = (float)v;
            im = 0.0f;
        }
        size_t base = ((size_t)inf->isz * e->nrz_per_range + iz) * e->nrr + ir;
        cx->out->field[2 * base] += re;
        cx->out->field[2 * base + 1] += im;
    }
}

/* src/influence.hpp:91-100 */
static double adjust_sigma(const Ctx *cx, double sigma, const RayPt *p0, const RayPt *p1, const Infl *inf)
{
    if(!cx->gauss) return sigma;
    double lambda = p0->c / inf->freq0;
    return dmax(sigma, dmin(FLT(0.2) * inf->freq0 * creal(p1->tau), PI * lambda));
}

/* src/influence.hpp:383-417 */
static int at_caustic(const Infl *inf, double q)
{
    return (q <= 0.0 && inf->qOld > 0.0) || (q >= 0.0 && inf->qOld < 0.0);
}

/* src/influence.hpp:897-1024 (2-D branch) */
static void geo_core(Ctx *cx, double s, double n1, double dq, cpx dtau, int ir, int iz, int is,
                     const RayPt *p0, const RayPt *p1, double RcvrDecl, const Infl *inf)
{
    double qFinal = p0->q.x + s * dq;
    double sigma = fabs(qFinal * inf->rcp_q0), sigma_orig = sigma;
    sigma = adjust_sigma(cx, sigma, p0, p1, inf);
    double bcd = n1;
    if(bcd > inf->BeamWindow * sigma || bcd == inf->BeamWindow * sigma) return;
    cpx delay = p0->tau + s * dtau;
    double cfactor = sqrt(p1->c);
    double cnst = inf->Ratio1 * cfactor * p1->Amp / sqrt(fabs(qFinal));
    double w;
    if(cx->gauss) w = exp(FLT(-0.5) * (n1 / sigma) * (n1 / sigma)) * (sigma_orig / sigma);
    else w = (sigma - n1) / sigma;
    const RayPt *pp = cx->gauss ? p1 : p0;
    double phaseInt = pp->Phase + inf->phase;
    if(at_caustic(inf, qFinal)) phaseInt = inf->phase + PI / FLT(2.0);
    apply_contrib(cx, cnst, w, inf->omega, delay, phaseInt, RcvrDecl, ir, iz, is, inf, p1);
}

/* src/influence.hpp:1201-1406 (2-D branch) */
static void step_infl_geocart(Ctx *cx, const RayPt *p0, const RayPt *p1, Infl *inf, int is)
{
    const Env *e = cx->e;
    double rA = inf->x.x, rB = p1->x.x;
    v2 xray = p0->x;
    v2 rayt = vsub(p1->x, p0->x);
    double rlen = vlen(rayt);
    if(rlen < 1.0e3 * spacing(p1->x.x)) return; /* IsSmallValue, const_thresh false */
    rayt = vdiv(rayt, rlen);
    v2 rayn = V(-rayt.y, rayt.x);
    double RcvrDecl = RAD_DEG * atan2(rayt.y, rayt.x);
    double dq = p1->q.x - p0->q.x;
    cpx dtau = p1->tau - p0->tau;
    double phaseq = p0->q.x;
    if(at_caustic(inf, phaseq)) inf->phase += PI / FLT(2.0);
    inf->qOld = phaseq;
    double sigma = dmax(fabs(p0->q.x), fabs(p1->q.x)) * inf->rcp_q0 / fabs(rayt.x);
    sigma = adjust_sigma(cx, sigma, p0, p1, inf);
    double RadiusMax = inf->BeamWindow * sigma, zmin, zmax;
    if(fabs(rayt.x) > FLT(0.50001)) {
        zmin = dmin(p0->x.y, p1->x.y) - RadiusMax;
        zmax = dmax(p0->x.y, p1->x.y) + RadiusMax;
    } else {
        zmin = -DBL_MAX;
        zmax = DBL_MAX;
    }
    for(;;) {
        double rr = e->rr[inf->ir];
        if(rr >= dmin(rA, rB) && rr < dmax(rA, rB)) {
            for(int iz = 0; iz < e->nrz_per_range; ++iz) {
                int tiz = (e->run_type[4] == 'I') ? inf->ir : iz;
                double zr = e->rz[tiz];
                if(zr < zmin || zr > zmax) continue;
                v2 d = V(rr - xray.x, zr - xray.y);
                double s = vdot(d, rayt) / rlen;
                double n1 = fabs(vdot(d, rayn));
                geo_core(cx, s, n1, dq, dtau, inf->ir, iz, is, p0, p1, RcvrDecl, inf);
            }
        }
        int irTT;
        if(rB > e->rr[inf->ir]) {
            if(inf->ir >= e->nrr - 1) break;
            irTT = inf->ir + 1;
            if(e->rr[irTT] >= rB) break;
        } else {
            if(inf->ir <= 0) break;
            irTT = inf->ir - 1;
            if(e->rr[irTT] <= rB) break;
        }
        inf->ir = irTT;
    }
    inf->x = p1->x;
}

/* ------------------------------------------------------------------ */
/* per-ray driver: src/trace.hpp:76-266 (RayInit), 274-381 (RayUpdate),  */
/* 391-477 (RayTerminate), 525-589 (MainFieldModes)                     */
/* ------------------------------------------------------------------ */
static void trace_ray(Ctx *cx, int isz, int ialpha, ErrSt *err)
{
    const Env *e = cx->e;
    SegSt iSeg = {0, 0};
    RayPt p0, p1, p2;
    memset(&p0, 0, sizeof(p0));
    memset(&p1, 0, sizeof(p1));
    memset(&p2, 0, sizeof(p2));
    double alpha = e->alpha[ialpha];
    double SrcDecl = RAD_DEG * alpha;
    v2 xs = V(FLT(0.0), (double)e->sz[isz]);
    v2 tinit = V(cos(alpha), sin(alpha));
    SSPOut o;
    eval_ssp(xs, tinit, &o, e, &iSeg, err);
    double c = creal(o.ccpx);
    {   /* too-few-beams warning (trace.hpp:119-134) */
        double dopt = sqrt(c / (FLT(6.0) * e->freq0 * e->rr[e->nrr - 1]));
        int nopt = 2 + (int)((e->alpha[e->nalpha - 1] - e->alpha[0]) / dopt);
        if(cx->coherent && e->nalpha < nopt && ialpha == 0) run_warn(err, W_TOO_FEW);
    }
    int ibp = bsearch_leq(e->sbp, e->nsbp, 2, 0, SrcDecl);
    ibp = imin(ibp, e->nsbp - 2);
    double s = (SrcDecl - e->sbp[2 * ibp]) / (e->sbp[2 * (ibp + 1)] - e->sbp[2 * ibp]);
    float Amp0 = (float)((FLT(1.0) - s) * e->sbp[2 * ibp + 1] + s * e->sbp[2 * (ibp + 1) + 1]);
    if(e->run_type[0] == 'S') {
        float om = (float)(FLT(2.0) * PI * e->freq0);
        Amp0 = (float)(Amp0 * ((double)sqrtf(2.0f) * fabs(sin(om / c * xs.y * sin(alpha)))));
    }
    p0.x = xs;
    p0.c = c;
    p0.t = vdiv(tinit, c);
    p0.tau = 0.0;
    p0.Amp = Amp0;
    p0.Phase = 0.0;
    p0.p = V(1.0, 0.0);
    p0.q = V(0.0, 1.0);
    if(e->run_type[1] == 'G') p0.q = V(0.0, 0.0);
    HS htop = e->top, hbot = e->bot;
    BdSt top, bot;
    memset(&top, 0, sizeof(top));
    memset(&bot, 0, sizeof(bot));
    get_bdry_seg(xs, p0.t, &top, &e->btop, &htop, 1, 1, err);
    get_bdry_seg(xs, p0.t, &bot, &e->bbot, &hbot, 0, 1, err);
    double dBegTop, dBegBot, dEndTop, dEndBot;
    distances(xs, &top, &bot, &dBegTop, &dBegBot);
    if(dBegTop <= 0.0 || dBegBot <= 0.0) {
        run_warn(err, W_SRC_OUTSIDE);
        return;
    }
    /* Init_Influence src/influence.hpp:525-644 */
    Infl inf;
    memset(&inf, 0, sizeof(inf));
    inf.isz = isz;
    inf.ialpha = ialpha;
    inf.alpha = alpha;
    inf.SrcDeclAngle = SrcDecl;
    inf.freq0 = e->freq0;
    inf.omega = FLT(2.0) * PI * inf.freq0;
    inf.c0 = p0.c;
    inf.RadMax = FLT(50.0) * p0.c / e->freq0;
    inf.BeamWindow = cx->gauss ? 4.0 : 1.0;
    inf.Ratio1 = sqrt(fabs(cos(alpha)));
    if(e->run_type[3] == 'X') inf.Ratio1 = 1.0;
    if(cx->gauss) inf.Ratio1 /= sqrt(FLT(2.0) * PI);
    inf.rcp_q0 = e->dalpha / p0.c;
    inf.phase = FLT(0.0);
    inf.qOld = p0.q.x;
    inf.x = p0.x;
    inf.ir = bsearch_gt(e->rr, e->nrr, p0.x.x);
    if(p0.t.x < 0.0 && inf.ir > 0) --inf.ir;

    int small = 0, is = 0;
    for(;;) {
        if(err->err) break;
        int trefl = 0, brefl = 0;
        step2d(p0, &p1, &top, &bot, e, &iSeg, err, &small, &trefl, &brefl);
        cx->out->nsteps++;
        get_bdry_seg(p1.x, p1.t, &top, &e->btop, &htop, 1, 0, err);
        get_bdry_seg(p1.x, p1.t, &bot, &e->bbot, &hbot, 0, 0, err);
        distances(p1.x, &top, &bot, &dEndTop, &dEndBot);
        int two = 0;
        if(trefl || brefl) {
            const Bdry *bdi = trefl ? &e->btop : &e->bbot;
            const BdSt *bst = trefl ? &top : &bot;
            const HS *hs = trefl ? &htop : &hbot;
            const BdPt *b0 = &bdi->bd[bst->Iseg], *b1 = b0 + 1;
            v2 nInt, tInt;
            if(bdi->type[0] == 'C') {
                double sss = vdot(vsub(p1.x, bst->x), b0->t) / b0->Len;
                nInt = vadd(vsc(FLT(1.0) - sss, b0->Noden), vsc(sss, b1->Noden));
                tInt = vadd(vsc(FLT(1.0) - sss, b0->Nodet), vsc(sss, b1->Nodet));
            } else {
                nInt = b0->n;
                tInt = b0->t;
            }
            reflect2d(p1, &p2, hs, trefl, tInt, nInt, b0->kappa, e, &iSeg, err);
            distances(p2.x, &top, &bot, &dEndTop, &dEndBot);
            two = 1;
        }
        step_infl_geocart(cx, &p0, &p1, &inf, is);
        ++is;
        if(two) {
            step_infl_geocart(cx, &p1, &p2, &inf, is);
            p0 = p2;
            ++is;
        } else {
            p0 = p1;
        }
        /* RayTerminate */
        int leftbox = outside_box(p0.x, e, 0) || outside_box(p0.x, e, 1);
        int escaped = (dBegTop < 0.0 && dEndTop < 0.0) || (dBegBot < 0.0 && dEndBot < 0.0);
        int lost = p0.Amp < FLT(0.005);
        if(leftbox || lost || escaped) break;
        if(is >= MAXN - 3) {
            run_warn(err, W_ONERAY_MEM);
            break;
        }
        dBegTop = dEndTop;
        dBegBot = dEndBot;
    }
}

int oracle2d_sizes(const O2Env *env, O2Out *out)
{
    Env e;
    int r = build_env(env, &e, out);
    free_env(&e);
    return r;
}

/* src/influence.hpp:1556-1627 (2-D ScalePressure) and src/mode/arr.cpp:24-74 */
static void postprocess(Ctx *cx)
{
    const Env *e = cx->e;
    O2Out *o = cx->out;
    int ntot = e->nsz * e->nrz_per_range;
    if(cx->tl && o->field) {
        double cnst = FLT(-1.0);
        for(int k = 0; k < ntot; ++k) {
            for(int ir = 0; ir < e->nrr; ++ir) {
                float *u = &o->field[2 * ((size_t)k * e->nrr + ir)];
                if(!cx->coherent) { u[0] = sqrtf(u[0]); u[1] = 0.0f; }
                double factor;
                if(e->run_type[3] == 'X') factor = (double)(-4.0f * sqrtf(3.14159265f)) * cnst;
                else if(fabs(e->rr[ir]) < REAL_EPS) factor = 0.0;
                else factor = cnst / sqrt(fabs(e->rr[ir]));
                u[0] *= (float)factor;
                u[1] *= (float)factor;
            }
        }
    }
    if(cx->arrivals && o->narr) {
        for(int k = 0; k < ntot; ++k) {
            for(int ir = 0; ir < e->nrr; ++ir) {
                size_t base = (size_t)k * e->nrr + ir;
                int narr = o->narr[base];
                if(narr > e->max_narr) o->narr[base] = narr = e->max_narr;
                float factor;
                if(e->run_type[3] == 'X') factor = (float)(FLT(4.0) * sqrt(PI));
                else if(fabs(e->rr[ir]) < REAL_EPS) factor = FLT(1e5);
                else factor = (float)(FLT(1.0) / sqrt(e->rr[ir]));
                for(int a = 0; a < narr; ++a) o->arr[base * e->max_narr + a].a *= factor;
            }
        }
    }
}

int oracle2d_run(const O2Env *env, O2Out *out)
{
    Env e;
    if(build_env(env, &e, out) != 0) { free_env(&e); return -1; }
    Ctx cx;
    memset(&cx, 0, sizeof(cx));
    cx.e = &e;
    cx.out = out;
    char rt = e.run_type[0];
    cx.gauss = (e.beam_type[0] == 'B' || e.beam_type[0] == 'b');
    cx.coherent = rt == 'C';
    cx.tl = rt == 'C' || rt == 'S' || rt == 'I';
    cx.arrivals = rt == 'A' || rt == 'a' || rt == 'V' || rt == 'v';
    cx.also_eigen = rt == 'V' || rt == 'v';
    cx.eigen = rt == 'E';
    char bt = e.beam_type[0];
    if(!(bt == 'G' || bt == 'B' || bt == '^' || bt == ' ')) { free_env(&e); return -2; }
    out->nsteps = out->nevals = 0;
    out->neigen = 0;
    if(out->rr_m) memcpy(out->rr_m, e.rr, e.nrr * sizeof(double));
    if(out->rz_m) memcpy(out->rz_m, e.rz, e.nrz * sizeof(float));
    if(out->alpha_rad) memcpy(out->alpha_rad, e.alpha, e.nalpha * sizeof(double));
    ErrSt err = {0, 0};
    /* job order of GetJobIndices (src/common.hpp:365-391): ialpha fastest */
    int nalpha = (e.isingle > 0) ? 1 : e.nalpha;
    int njobs = nalpha * e.nsz;
    int j0 = 0, j1 = njobs;
    if(out->ray_count > 0) {
        j0 = out->ray_first;
        j1 = imin(njobs, out->ray_first + out->ray_count);
    }
    for(int job = j0; job < j1; ++job) {
        int ia = (e.isingle > 0) ? e.isingle - 1 : job % nalpha;
        int isz = job / nalpha;
        trace_ray(&cx, isz, ia, &err);
        if(err.err) break;
    }
    postprocess(&cx);
    out->err_bits = err.err;
    out->warn_bits = err.warn;
    free_env(&e);
    return err.err ? 1 : 0;
}
