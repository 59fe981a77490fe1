/* TEST INFRASTRUCTURE ONLY — the CPU oracle (see svsim_oracle.h).
 *
 * Every function restates one piece of the reference and cites it.  Line numbers
 * refer to svsim/src/svsim_nvgpu_sin.cuh unless another file is named; the CPU
 * twin svsim/src/svsim_cpu_sin.hpp carries the same expressions (:602-1165 and
 * :2103-2460).  The arithmetic of each gate is written in the same evaluation
 * order as the reference (left-associated sums of products), and the file is
 * built with -ffp-contract=off, so on x86-64 it reproduces the reference CPU
 * backend bit for bit; tests/test_oracle.py checks exactly that.
 */
#include "svsim_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OR_PI  3.14159265358979323846   /* config.hpp:52 */
#define OR_S2I 0.70710678118654752440   /* config.hpp:54 */

enum {
    U3, U2, U1, CX, ID, X, Y, Z, H, S,
    SDG, T, TDG, RX, RY, RZ, CZ, CY, SWAP, CH,
    CCX, CSWAP, CRX, CRY, CRZ, CU1, CU3, RXX, RZZ, RCCX,
    RC3X, C3X, C3SQRTX, C4X, R, SRN, W, RYY, N_OPS
};

typedef struct { uint32_t n; double* re; double* im; } sv_t;

/* Pair enumeration of OP_HEAD (:640-648): i in [0, 2^(n-1)),
 * pos0 = ((i >> q) << (q+1)) + (i & (2^q - 1)), pos1 = pos0 + 2^q. */
#define PAIR_LOOP_BEGIN(sv, q)                                              \
    {                                                                       \
        const uint64_t half_ = (uint64_t)1 << ((sv)->n - 1);                \
        const uint64_t qd_ = (uint64_t)1 << (q);                            \
        double* const re_ = (sv)->re;                                       \
        double* const im_ = (sv)->im;                                       \
        _Pragma("omp parallel for schedule(static) if (half_ >= 65536)")    \
        for (uint64_t i = 0; i < half_; i++) {                              \
            const uint64_t pos0 = ((i >> (q)) << ((q) + 1)) + (i & (qd_ - 1)); \
            const uint64_t pos1 = pos0 + qd_;                               \
            const double a0r = re_[pos0], a0i = im_[pos0];                  \
            const double a1r = re_[pos1], a1i = im_[pos1];                  \
            (void)a0r; (void)a0i; (void)a1r; (void)a1i;
#define PAIR_LOOP_END }}

/* C1_GATE :654-675 — general 2x2 complex matrix. */
static void g_c1(sv_t* sv, double e0r, double e0i, double e1r, double e1i,
                 double e2r, double e2i, double e3r, double e3i, uint32_t q)
{
    PAIR_LOOP_BEGIN(sv, q)
        re_[pos0] = (e0r * a0r) - (e0i * a0i) + (e1r * a1r) - (e1i * a1i);
        im_[pos0] = (e0r * a0i) + (e0i * a0r) + (e1r * a1i) + (e1i * a1r);
        re_[pos1] = (e2r * a0r) - (e2i * a0i) + (e3r * a1r) - (e3i * a1i);
        im_[pos1] = (e2r * a0i) + (e2i * a0r) + (e3r * a1i) + (e3i * a1r);
    PAIR_LOOP_END
}

/* CX_GATE :779-811 — swap the (ctrl=1, target=0) and (ctrl=1, target=1)
 * amplitudes.  Each quad is independent, so the visiting order is free; this
 * enumerates the 2^(n-2) quads by inserting zero bits at both positions. */
static void g_cx(sv_t* sv, uint32_t c, uint32_t t)
{
    const uint32_t lo = c < t ? c : t, hi = c < t ? t : c;
    const uint64_t quarter = (uint64_t)1 << (sv->n - 2);
    const uint64_t cd = (uint64_t)1 << c, td = (uint64_t)1 << t;
    double* const re = sv->re;
    double* const im = sv->im;
    #pragma omp parallel for schedule(static) if (quarter >= 65536)
    for (uint64_t i = 0; i < quarter; i++) {
        uint64_t b = i;
        b = ((b >> lo) << (lo + 1)) | (b & (((uint64_t)1 << lo) - 1));
        b = ((b >> hi) << (hi + 1)) | (b & (((uint64_t)1 << hi) - 1));
        const uint64_t p0 = b | cd, p1 = b | cd | td;
        const double r0 = re[p0], i0 = im[p0];
        re[p0] = re[p1]; im[p0] = im[p1];
        re[p1] = r0;     im[p1] = i0;
    }
}

/* X_GATE :818-830 */
static void g_x(sv_t* sv, uint32_t q)
{
    PAIR_LOOP_BEGIN(sv, q)
        re_[pos0] = a1r; im_[pos0] = a1i;
        re_[pos1] = a0r; im_[pos1] = a0i;
    PAIR_LOOP_END
}
/* Y_GATE :837-850 */
static void g_y(sv_t* sv, uint32_t q)
{
    PAIR_LOOP_BEGIN(sv, q)
        re_[pos0] = a1i;  im_[pos0] = -a1r;
        re_[pos1] = -a0i; im_[pos1] = a0r;
    PAIR_LOOP_END
}
/* Z_GATE :857-866 */
static void g_z(sv_t* sv, uint32_t q)
{
    PAIR_LOOP_BEGIN(sv, q)
        re_[pos1] = -a1r; im_[pos1] = -a1i;
    PAIR_LOOP_END
}
/* H_GATE :873-887 */
static void g_h(sv_t* sv, uint32_t q)
{
    PAIR_LOOP_BEGIN(sv, q)
        re_[pos0] = OR_S2I * (a0r + a1r); im_[pos0] = OR_S2I * (a0i + a1i);
        re_[pos1] = OR_S2I * (a0r - a1r); im_[pos1] = OR_S2I * (a0i - a1i);
    PAIR_LOOP_END
}
/* SRN_GATE :894-907 (as coded: not a square root of X, and not unitary) */
static void g_srn(sv_t* sv, uint32_t q)
{
    PAIR_LOOP_BEGIN(sv, q)
        re_[pos0] = 0.5 * (a0r + a1r);  im_[pos0] = 0.5 * (a0i - a1i);
        re_[pos1] = 0.5 * (a0r + a1r);  im_[pos1] = 0.5 * (-a0i + a1i);
    PAIR_LOOP_END
}
/* R_GATE :924-933 (as coded: multiplies |1> by i*phase) */
static void g_r(sv_t* sv, double phase, uint32_t q)
{
    PAIR_LOOP_BEGIN(sv, q)
        re_[pos1] = -(a1i * phase); im_[pos1] = a1r * phase;
    PAIR_LOOP_END
}
/* S_GATE :940-948 */
static void g_s(sv_t* sv, uint32_t q)
{
    PAIR_LOOP_BEGIN(sv, q)
        re_[pos1] = -a1i; im_[pos1] = a1r;
    PAIR_LOOP_END
}
/* SDG_GATE :955-963 */
static void g_sdg(sv_t* sv, uint32_t q)
{
    PAIR_LOOP_BEGIN(sv, q)
        re_[pos1] = a1i; im_[pos1] = -a1r;
    PAIR_LOOP_END
}
/* T_GATE :970-978 */
static void g_t(sv_t* sv, uint32_t q)
{
    PAIR_LOOP_BEGIN(sv, q)
        re_[pos1] = OR_S2I * (a1r - a1i); im_[pos1] = OR_S2I * (a1r + a1i);
    PAIR_LOOP_END
}
/* TDG_GATE :985-993 */
static void g_tdg(sv_t* sv, uint32_t q)
{
    PAIR_LOOP_BEGIN(sv, q)
        re_[pos1] = OR_S2I * (a1r + a1i); im_[pos1] = OR_S2I * (-a1r + a1i);
    PAIR_LOOP_END
}
/* U1_GATE :1022-1038 (pos0 is rewritten unchanged, pos1 gets e^{i lambda}) */
static void g_u1(sv_t* sv, double lambda, uint32_t q)
{
    const double e3r = cos(lambda), e3i = sin(lambda);
    PAIR_LOOP_BEGIN(sv, q)
        re_[pos1] = (e3r * a1r) - (e3i * a1i);
        im_[pos1] = (e3r * a1i) + (e3i * a1r);
    PAIR_LOOP_END
}
/* U2_GATE :1045-1059 */
static void g_u2(sv_t* sv, double phi, double lambda, uint32_t q)
{
    g_c1(sv, OR_S2I, 0, -OR_S2I * cos(lambda), -OR_S2I * sin(lambda),
         OR_S2I * cos(phi), OR_S2I * sin(phi),
         OR_S2I * cos(phi + lambda), OR_S2I * sin(phi + lambda), q);
}
/* U3_GATE :1066-1081 */
static void g_u3(sv_t* sv, double theta, double phi, double lambda, uint32_t q)
{
    g_c1(sv, cos(theta / 2.), 0,
         -cos(lambda) * sin(theta / 2.), -sin(lambda) * sin(theta / 2.),
         cos(phi) * sin(theta / 2.), sin(phi) * sin(theta / 2.),
         cos(phi + lambda) * cos(theta / 2.), sin(phi + lambda) * cos(theta / 2.), q);
}
/* RX_GATE :1085-1100 */
static void g_rx(sv_t* sv, double theta, uint32_t q)
{
    const double rxr = cos(theta / 2.0), rxi = -sin(theta / 2.0);
    PAIR_LOOP_BEGIN(sv, q)
        re_[pos0] = (rxr * a0r) - (rxi * a1i);
        im_[pos0] = (rxr * a0i) + (rxi * a1r);
        re_[pos1] = -(rxi * a0i) + (rxr * a1r);
        im_[pos1] = +(rxi * a0r) + (rxr * a1i);
    PAIR_LOOP_END
}
/* RY_GATE :1104-1122 */
static void g_ry(sv_t* sv, double theta, uint32_t q)
{
    const double e0r = cos(theta / 2.0), e1r = -sin(theta / 2.0);
    const double e2r = sin(theta / 2.0), e3r = cos(theta / 2.0);
    PAIR_LOOP_BEGIN(sv, q)
        re_[pos0] = (e0r * a0r) + (e1r * a1r);
        im_[pos0] = (e0r * a0i) + (e1r * a1i);
        re_[pos1] = (e2r * a0r) + (e3r * a1r);
        im_[pos1] = (e2r * a0i) + (e3r * a1i);
    PAIR_LOOP_END
}
/* W_GATE :1428-1440 */
static void g_w(sv_t* sv, uint32_t q)
{
    PAIR_LOOP_BEGIN(sv, q)
        re_[pos0] = OR_S2I * (a0r + a1i);  im_[pos0] = OR_S2I * (a0i - a1r);
        re_[pos1] = OR_S2I * (a0i + a1r);  im_[pos1] = OR_S2I * (-a0r + a1i);
    PAIR_LOOP_END
}

/* ---- composites :1134-1454, same elementary sequences as the reference ---- */
static void g_cu1(sv_t* sv, double l, uint32_t a, uint32_t b)   /* CU1_GATE :1183-1193 */
{
    g_u1(sv, l / 2, a); g_cx(sv, a, b); g_u1(sv, -l / 2, b); g_cx(sv, a, b); g_u1(sv, l / 2, b);
}
static void g_ccx(sv_t* sv, uint32_t a, uint32_t b, uint32_t c) /* CCX_GATE :1211-1230 */
{
    g_h(sv, c);  g_cx(sv, b, c); g_tdg(sv, c); g_cx(sv, a, c); g_t(sv, c);
    g_cx(sv, b, c); g_tdg(sv, c); g_cx(sv, a, c); g_t(sv, b); g_t(sv, c);
    g_h(sv, c);  g_cx(sv, a, b); g_t(sv, a); g_tdg(sv, b); g_cx(sv, a, b);
}
static void g_c3x_like(sv_t* sv, double ang, uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{   /* C3X_GATE :1339-1370 with ang = PI/4; C3SQRTX_GATE :1374-1404 with ang = PI/8 */
    g_h(sv, d); g_cu1(sv, -ang, a, d); g_h(sv, d);
    g_cx(sv, a, b);
    g_h(sv, d); g_cu1(sv, ang, b, d); g_h(sv, d);
    g_cx(sv, a, b);
    g_h(sv, d); g_cu1(sv, -ang, b, d); g_h(sv, d);
    g_cx(sv, b, c);
    g_h(sv, d); g_cu1(sv, ang, c, d); g_h(sv, d);
    g_cx(sv, a, c);
    g_h(sv, d); g_cu1(sv, -ang, c, d); g_h(sv, d);
    g_cx(sv, b, c);
    g_h(sv, d); g_cu1(sv, ang, c, d); g_h(sv, d);
    g_cx(sv, a, c);
    g_h(sv, d); g_cu1(sv, -ang, c, d); g_h(sv, d);
}

int oracle_apply_gate(uint32_t n, const oracle_gate* g, double* re, double* im)
{
    sv_t s = { n, re, im };
    sv_t* sv = &s;
    const uint32_t* q = g->qb;
    const double th = g->theta, ph = g->phi, la = g->lambda;
    /* parameter fields follow the *_OP wrappers :1459-1647 */
    switch (g->op) {
    case U3:  g_u3(sv, th, ph, la, q[0]); break;
    case U2:  g_u2(sv, ph, la, q[0]); break;
    case U1:  g_u1(sv, la, q[0]); break;
    case CX:  g_cx(sv, q[0], q[1]); break;
    case ID:  break;                                               /* :913-917 */
    case X:   g_x(sv, q[0]); break;
    case Y:   g_y(sv, q[0]); break;
    case Z:   g_z(sv, q[0]); break;
    case H:   g_h(sv, q[0]); break;
    case S:   g_s(sv, q[0]); break;
    case SDG: g_sdg(sv, q[0]); break;
    case T:   g_t(sv, q[0]); break;
    case TDG: g_tdg(sv, q[0]); break;
    case RX:  g_rx(sv, th, q[0]); break;
    case RY:  g_ry(sv, th, q[0]); break;
    case RZ:  g_u1(sv, ph, q[0]); break;                           /* RZ_GATE :1126-1130 */
    case CZ:  g_h(sv, q[1]); g_cx(sv, q[0], q[1]); g_h(sv, q[1]); break;       /* CZ_GATE :1134-1140 */
    case CY:  g_sdg(sv, q[1]); g_cx(sv, q[0], q[1]); g_s(sv, q[1]); break;     /* CY_GATE :1144-1150 */
    case SWAP: g_cx(sv, q[0], q[1]); g_cx(sv, q[1], q[0]); g_cx(sv, q[0], q[1]); break; /* SWAP_GATE :1232-1238 */
    case CH: {                                                     /* CH_GATE :1154-1168 */
        const uint32_t a = q[0], b = q[1];
        g_h(sv, b); g_sdg(sv, b); g_cx(sv, a, b); g_h(sv, b); g_t(sv, b);
        g_cx(sv, a, b); g_t(sv, b); g_h(sv, b); g_s(sv, b); g_x(sv, b); g_s(sv, a);
        break; }
    case CCX: g_ccx(sv, q[0], q[1], q[2]); break;
    case CSWAP:                                                    /* CSWAP_GATE :1241-1247 */
        g_cx(sv, q[2], q[1]); g_ccx(sv, q[0], q[1], q[2]); g_cx(sv, q[2], q[1]); break;
    case CRX: {                                                    /* CRX_GATE :1251-1259 */
        const uint32_t a = q[0], b = q[1];
        g_u1(sv, OR_PI / 2, b); g_cx(sv, a, b); g_u3(sv, -la / 2, 0, 0, b);
        g_cx(sv, a, b); g_u3(sv, la / 2, -OR_PI / 2, 0, b);
        break; }
    case CRY: {                                                    /* CRY_GATE :1263-1270 */
        const uint32_t a = q[0], b = q[1];
        g_u3(sv, la / 2, 0, 0, b); g_cx(sv, a, b); g_u3(sv, -la / 2, 0, 0, b); g_cx(sv, a, b);
        break; }
    case CRZ: {                                                    /* CRZ_GATE :1172-1179 */
        const uint32_t a = q[0], b = q[1];
        g_u1(sv, la / 2, b); g_cx(sv, a, b); g_u1(sv, -la / 2, b); g_cx(sv, a, b);
        break; }
    case CU1: g_cu1(sv, la, q[0], q[1]); break;
    case CU3: {                                                    /* CU3_GATE :1195-1207 */
        const uint32_t c = q[0], t = q[1];
        const double temp1 = (la - ph) / 2, temp2 = th / 2, temp3 = -(ph + la) / 2;
        g_u1(sv, -temp3, c); g_u1(sv, temp1, t); g_cx(sv, c, t);
        g_u3(sv, -temp2, 0, temp3, t); g_cx(sv, c, t); g_u3(sv, temp2, ph, 0, t);
        break; }
    case RXX: {                                                    /* RXX_GATE :1274-1284 */
        const uint32_t a = q[0], b = q[1];
        g_u3(sv, OR_PI / 2, th, 0, a); g_h(sv, b); g_cx(sv, a, b); g_u1(sv, -th, b);
        g_cx(sv, a, b); g_h(sv, b); g_u2(sv, -OR_PI, OR_PI - th, a);
        break; }
    case RZZ: g_cx(sv, q[0], q[1]); g_u1(sv, th, q[1]); g_cx(sv, q[0], q[1]); break; /* RZZ_GATE :1288-1294 */
    case RCCX: {                                                   /* RCCX_GATE :1298-1310 */
        const uint32_t a = q[0], b = q[1], c = q[2];
        g_u2(sv, 0, OR_PI, c); g_u1(sv, OR_PI / 4, c); g_cx(sv, b, c); g_u1(sv, -OR_PI / 4, c);
        g_cx(sv, a, c); g_u1(sv, OR_PI / 4, c); g_cx(sv, b, c); g_u1(sv, -OR_PI / 4, c);
        g_u2(sv, 0, OR_PI, c);
        break; }
    case RC3X: {                                                   /* RC3X_GATE :1314-1335 */
        const uint32_t a = q[0], b = q[1], c = q[2], d = q[3];
        g_u2(sv, 0, OR_PI, d); g_u1(sv, OR_PI / 4, d); g_cx(sv, c, d); g_u1(sv, -OR_PI / 4, d);
        g_u2(sv, 0, OR_PI, d); g_cx(sv, a, d); g_u1(sv, OR_PI / 4, d); g_cx(sv, b, d);
        g_u1(sv, -OR_PI / 4, d); g_cx(sv, a, d); g_u1(sv, OR_PI / 4, d); g_cx(sv, b, d);
        g_u1(sv, -OR_PI / 4, d); g_u2(sv, 0, OR_PI, d); g_u1(sv, OR_PI / 4, d); g_cx(sv, c, d);
        g_u1(sv, -OR_PI / 4, d); g_u2(sv, 0, OR_PI, d);
        break; }
    case C3X:     g_c3x_like(sv, OR_PI / 4, q[0], q[1], q[2], q[3]); break;
    case C3SQRTX: g_c3x_like(sv, OR_PI / 8, q[0], q[1], q[2], q[3]); break;
    case C4X: {                                                    /* C4X_GATE :1408-1420 */
        const uint32_t a = q[0], b = q[1], c = q[2], d = q[3], e = q[4];
        g_h(sv, e); g_cu1(sv, -OR_PI / 2, d, e); g_h(sv, e);
        g_c3x_like(sv, OR_PI / 4, a, b, c, d);
        g_h(sv, d); g_cu1(sv, OR_PI / 4, d, e); g_h(sv, d);
        g_c3x_like(sv, OR_PI / 4, a, b, c, d);
        g_c3x_like(sv, OR_PI / 8, a, b, c, e);
        break; }
    case R:   g_r(sv, th, q[0]); break;
    case SRN: g_srn(sv, q[0]); break;
    case W:   g_w(sv, q[0]); break;
    case RYY: {                                                    /* RYY_GATE :1444-1454 */
        const uint32_t a = q[0], b = q[1];
        g_rx(sv, OR_PI / 2, a); g_rx(sv, OR_PI / 2, b); g_cx(sv, a, b); g_u1(sv, th, b);
        g_cx(sv, a, b); g_rx(sv, -OR_PI / 2, a); g_rx(sv, -OR_PI / 2, b);
        break; }
    default: return -1;
    }
    return 0;
}

/* Simulation ctor / reset_sv :193-255 */
void oracle_reset(uint32_t n, double* re, double* im)
{
    const uint64_t dim = (uint64_t)1 << n;
    memset(re, 0, dim * sizeof(double));
    memset(im, 0, dim * sizeof(double));
    re[0] = 1.0;
}

int oracle_apply(uint32_t n, const oracle_gate* gates, size_t n_gates, double* re, double* im)
{
    for (size_t t = 0; t < n_gates; t++)          /* simulation_kernel :614-621 */
        if (oracle_apply_gate(n, &gates[t], re, im) != 0) return -1;
    return 0;
}

int oracle_run(uint32_t n, const oracle_gate* gates, size_t n_gates, double* re, double* im)
{
    oracle_reset(n, re, im);
    return oracle_apply(n, gates, n_gates, re, im);
}

/* Simulation::measure :359-383.  The scan is the reference's sequential
 * inclusive sum; a shot draws r and keeps the j with scan[j] <= r < scan[j+1],
 * or 0 if there is none.  The scan is non-decreasing, so that j is found by a
 * binary search for the first scan entry above r (same result, O(log dim)). */
void oracle_measure_uniforms(uint32_t n, const double* re, const double* im,
                             const double* uniforms, uint32_t shots, uint64_t* out, double* total)
{
    const uint64_t dim = (uint64_t)1 << n;
    double* scan = (double*)malloc((dim + 1) * sizeof(double));
    scan[0] = 0;
    for (uint64_t i = 1; i < dim + 1; i++)
        scan[i] = scan[i - 1] + ((re[i - 1] * re[i - 1]) + (im[i - 1] * im[i - 1]));
    for (uint32_t s = 0; s < shots; s++) {
        const double r = uniforms[s];
        uint64_t res = 0;
        if (scan[0] <= r && r < scan[dim]) {
            uint64_t lo = 0, hi = dim;      /* invariant: scan[lo] <= r < scan[hi] */
            while (hi - lo > 1) {
                const uint64_t mid = lo + (hi - lo) / 2;
                if (scan[mid] <= r) lo = mid; else hi = mid;
            }
            res = lo;
        }
        out[s] = res;
    }
    if (total) *total = scan[dim];
    free(scan);
}

double oracle_expectation(uint32_t n, const double* re, const double* im,
                          const oracle_pauli* terms, size_t n_terms)
{
    const uint64_t dim = (uint64_t)1 << n;
    double acc = 0;
    for (size_t t = 0; t < n_terms; t++) {
        const uint64_t xm = terms[t].x_mask, zm = terms[t].z_mask;
        const int ny = __builtin_popcountll(xm & zm) & 3;
        /* (P psi)[i] = i^ny (-1)^{popcount(j & zm)} psi[j], j = i ^ xm */
        double sr = 0, si = 0;
        for (uint64_t i = 0; i < dim; i++) {
            const uint64_t j = i ^ xm;
            double pr = re[j], pi = im[j];
            if (__builtin_popcountll(j & zm) & 1) { pr = -pr; pi = -pi; }
            double tr, ti;
            switch (ny) {
            case 0: tr = pr;  ti = pi;  break;
            case 1: tr = -pi; ti = pr;  break;
            case 2: tr = -pr; ti = -pi; break;
            default: tr = pi; ti = -pr; break;
            }
            /* conj(psi_i) * (P psi)_i */
            sr += re[i] * tr + im[i] * ti;
            si += re[i] * ti - im[i] * tr;
        }
        (void)si;
        acc += terms[t].coef * sr;
    }
    return acc;
}

int oracle_elementary_count(uint32_t op)
{
    /* Counted from the composite bodies :1134-1454 (ID = 0). */
    static const int counts[N_OPS] = {
        1, 1, 1, 1, 0, 1, 1, 1, 1, 1,
        1, 1, 1, 1, 1, 1, 3, 3, 3, 11,
        15, 17, 5, 4, 4, 5, 6, 7, 3, 9,
        18, 55, 55, 179, 1, 1, 1, 7 };
    return op < N_OPS ? counts[op] : -1;
}
