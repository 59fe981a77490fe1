// Lowering of reference gates into elementary ops.
//
// The reference applies each of its 38 ops as a fixed sequence of elementary gate
// sweeps (svsim/src/svsim_nvgpu_sin.cuh:1134-1454, one grid.sync each).  This file
// produces the same sequences, with every elementary matrix evaluated on the host
// by the reference's formulas, so each engine applies the reference's arithmetic
// gate for gate.  It also records, per elementary op, which of its angles depend on
// which angle field of the source gate (used by the adjoint).
#include <cmath>

#include "svb_internal.h"

namespace svb {
namespace {

constexpr double kPi = 3.14159265358979323846;    // config.hpp:52
constexpr double kS2I = 0.70710678118654752440;   // config.hpp:54

enum RefOp {
    U3, U2, U1, CX, ID, X, Y, Z, H, S,
    SDG, T, TDG, RX, RY, RZ, CZ, CY, SWAP, CH,
    CCX, CSWAP, CRX, CRY, CRZ, CU1, CU3, RXX, RZZ, RCCX,
    RC3X, C3X, C3SQRTX, C4X, R, SRN, W, RYY, N_REF_OPS
};

}  // namespace

// elementary kinds for the adjoint (EOp::kind)
enum { EK_CONST = 0, EK_U3 = 1, EK_U2 = 2, EK_U1 = 3, EK_RX = 4, EK_RY = 5, EK_R = 6 };

namespace {

struct Emitter {
    std::vector<EOp>& out;
    int32_t gate;

    EOp& push(uint8_t form, uint32_t q) {
        out.emplace_back();
        EOp& e = out.back();
        e.form = form;
        e.q = q;
        e.gate = gate;
        return e;
    }
    void fixed(uint8_t form, uint32_t q) { push(form, q); }
    void cx(uint32_t c, uint32_t t) { push(F_CX, t).c = c; }
    void x(uint32_t q) { fixed(F_X, q); }
    void h(uint32_t q) { fixed(F_H, q); }
    void s(uint32_t q) { fixed(F_S, q); }
    void sdg(uint32_t q) { fixed(F_SDG, q); }
    void t(uint32_t q) { fixed(F_T, q); }
    void tdg(uint32_t q) { fixed(F_TDG, q); }

    // U1_GATE :1022-1038.  dl[f] = d(lambda)/d(gate field f)
    void u1(double l, uint32_t q, double d0 = 0, double d1 = 0, double d2 = 0) {
        EOp& e = push(F_U1, q);
        e.m[0] = std::cos(l);
        e.m[1] = std::sin(l);
        e.kind = EK_U1;
        e.ang[2] = l;
        e.jac[2][0] = d0; e.jac[2][1] = d1; e.jac[2][2] = d2;
    }
    // U2_GATE :1045-1059
    void u2(double ph, double l, uint32_t q, const double dph[3], const double dl[3]) {
        EOp& e = push(F_C1, q);
        e.m[0] = kS2I;                 e.m[1] = 0;
        e.m[2] = -kS2I * std::cos(l);  e.m[3] = -kS2I * std::sin(l);
        e.m[4] = kS2I * std::cos(ph);  e.m[5] = kS2I * std::sin(ph);
        e.m[6] = kS2I * std::cos(ph + l);  e.m[7] = kS2I * std::sin(ph + l);
        e.kind = EK_U2;
        e.ang[1] = ph; e.ang[2] = l;
        for (int f = 0; f < 3; f++) { e.jac[1][f] = dph[f]; e.jac[2][f] = dl[f]; }
    }
    // U3_GATE :1066-1081
    void u3(double th, double ph, double l, uint32_t q, const double dth[3],
            const double dph[3], const double dl[3]) {
        EOp& e = push(F_C1, q);
        e.m[0] = std::cos(th / 2.);
        e.m[1] = 0;
        e.m[2] = -std::cos(l) * std::sin(th / 2.);
        e.m[3] = -std::sin(l) * std::sin(th / 2.);
        e.m[4] = std::cos(ph) * std::sin(th / 2.);
        e.m[5] = std::sin(ph) * std::sin(th / 2.);
        e.m[6] = std::cos(ph + l) * std::cos(th / 2.);
        e.m[7] = std::sin(ph + l) * std::cos(th / 2.);
        e.kind = EK_U3;
        e.ang[0] = th; e.ang[1] = ph; e.ang[2] = l;
        for (int f = 0; f < 3; f++) {
            e.jac[0][f] = dth[f]; e.jac[1][f] = dph[f]; e.jac[2][f] = dl[f];
        }
    }
    // RX_GATE :1085-1100
    void rx(double th, uint32_t q, double d0 = 0, double d1 = 0, double d2 = 0) {
        EOp& e = push(F_RX, q);
        e.m[0] = std::cos(th / 2.0);
        e.m[1] = -std::sin(th / 2.0);
        e.kind = EK_RX;
        e.ang[0] = th;
        e.jac[0][0] = d0; e.jac[0][1] = d1; e.jac[0][2] = d2;
    }
    // RY_GATE :1104-1122
    void ry(double th, uint32_t q, double d0 = 0) {
        EOp& e = push(F_RY, q);
        e.m[0] = std::cos(th / 2.0);
        e.m[1] = -std::sin(th / 2.0);
        e.m[2] = std::sin(th / 2.0);
        e.m[3] = std::cos(th / 2.0);
        e.kind = EK_RY;
        e.ang[0] = th;
        e.jac[0][0] = d0;
    }
    // CU1_GATE :1183-1193
    void cu1(double l, uint32_t a, uint32_t b, double dl2 = 0) {
        u1(l / 2, a, 0, 0, dl2 * 0.5);
        cx(a, b);
        u1(-l / 2, b, 0, 0, -dl2 * 0.5);
        cx(a, b);
        u1(l / 2, b, 0, 0, dl2 * 0.5);
    }
    // CCX_GATE :1211-1230
    void ccx(uint32_t a, uint32_t b, uint32_t c) {
        h(c); cx(b, c); tdg(c); cx(a, c); t(c); cx(b, c); tdg(c); cx(a, c);
        t(b); t(c); h(c); cx(a, b); t(a); tdg(b); cx(a, b);
    }
    // C3X_GATE :1339-1370 (ang = PI/4) and C3SQRTX_GATE :1374-1404 (ang = PI/8)
    void c3x_like(double ang, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
        h(d); cu1(-ang, a, d); h(d);
        cx(a, b);
        h(d); cu1(ang, b, d); h(d);
        cx(a, b);
        h(d); cu1(-ang, b, d); h(d);
        cx(b, c);
        h(d); cu1(ang, c, d); h(d);
        cx(a, c);
        h(d); cu1(-ang, c, d); h(d);
        cx(b, c);
        h(d); cu1(ang, c, d); h(d);
        cx(a, c);
        h(d); cu1(-ang, c, d); h(d);
    }
};

const double kZero3[3] = {0, 0, 0};

}  // namespace

bool lower_gate(const svb_gate& g, int32_t gate_index, std::vector<EOp>& out)
{
    Emitter em{out, gate_index};
    const uint32_t* q = g.qb;
    const double th = g.theta, ph = g.phi, la = g.lambda;
    const double dTH[3] = {1, 0, 0}, dPH[3] = {0, 1, 0}, dLA[3] = {0, 0, 1};
    switch (g.op) {
    case U3: em.u3(th, ph, la, q[0], dTH, dPH, dLA); break;
    case U2: em.u2(ph, la, q[0], dPH, dLA); break;
    case U1: em.u1(la, q[0], 0, 0, 1); break;
    case CX: em.cx(q[0], q[1]); break;
    case ID: break;                                       // ID_GATE :913-917
    case X:  em.x(q[0]); break;
    case Y:  em.fixed(F_Y, q[0]); break;
    case Z:  em.fixed(F_Z, q[0]); break;
    case H:  em.h(q[0]); break;
    case S:  em.s(q[0]); break;
    case SDG: em.sdg(q[0]); break;
    case T:  em.t(q[0]); break;
    case TDG: em.tdg(q[0]); break;
    case RX: em.rx(th, q[0], 1, 0, 0); break;
    case RY: em.ry(th, q[0], 1); break;
    case RZ: em.u1(ph, q[0], 0, 1, 0); break;             // RZ_GATE :1126-1130
    case CZ: em.h(q[1]); em.cx(q[0], q[1]); em.h(q[1]); break;          // :1134-1140
    case CY: em.sdg(q[1]); em.cx(q[0], q[1]); em.s(q[1]); break;        // :1144-1150
    case SWAP: em.cx(q[0], q[1]); em.cx(q[1], q[0]); em.cx(q[0], q[1]); break;  // :1232-1238
    case CH: {                                                          // :1154-1168
        const uint32_t a = q[0], b = q[1];
        em.h(b); em.sdg(b); em.cx(a, b); em.h(b); em.t(b); em.cx(a, b); em.t(b);
        em.h(b); em.s(b); em.x(b); em.s(a);
        break;
    }
    case CCX: em.ccx(q[0], q[1], q[2]); break;
    case CSWAP: em.cx(q[2], q[1]); em.ccx(q[0], q[1], q[2]); em.cx(q[2], q[1]); break;  // :1241-1247
    case CRX: {                                                         // :1251-1259
        const uint32_t a = q[0], b = q[1];
        const double dm[3] = {0, 0, -0.5}, dp[3] = {0, 0, 0.5};
        em.u1(kPi / 2, b);
        em.cx(a, b);
        em.u3(-la / 2, 0, 0, b, dm, kZero3, kZero3);
        em.cx(a, b);
        em.u3(la / 2, -kPi / 2, 0, b, dp, kZero3, kZero3);
        break;
    }
    case CRY: {                                                         // :1263-1270
        const uint32_t a = q[0], b = q[1];
        const double dm[3] = {0, 0, -0.5}, dp[3] = {0, 0, 0.5};
        em.u3(la / 2, 0, 0, b, dp, kZero3, kZero3);
        em.cx(a, b);
        em.u3(-la / 2, 0, 0, b, dm, kZero3, kZero3);
        em.cx(a, b);
        break;
    }
    case CRZ: {                                                         // :1172-1179
        const uint32_t a = q[0], b = q[1];
        em.u1(la / 2, b, 0, 0, 0.5);
        em.cx(a, b);
        em.u1(-la / 2, b, 0, 0, -0.5);
        em.cx(a, b);
        break;
    }
    case CU1: em.cu1(la, q[0], q[1], 1.0); break;
    case CU3: {                                                         // :1195-1207
        const uint32_t c = q[0], t = q[1];
        const double temp1 = (la - ph) / 2, temp2 = th / 2, temp3 = -(ph + la) / 2;
        em.u1(-temp3, c, 0, 0.5, 0.5);
        em.u1(temp1, t, 0, -0.5, 0.5);
        em.cx(c, t);
        const double a_th[3] = {-0.5, 0, 0}, a_la[3] = {0, -0.5, -0.5};
        em.u3(-temp2, 0, temp3, t, a_th, kZero3, a_la);
        em.cx(c, t);
        const double b_th[3] = {0.5, 0, 0};
        em.u3(temp2, ph, 0, t, b_th, dPH, kZero3);
        break;
    }
    case RXX: {                                                         // :1274-1284
        const uint32_t a = q[0], b = q[1];
        em.u3(kPi / 2, th, 0, a, kZero3, dTH, kZero3);
        em.h(b);
        em.cx(a, b);
        em.u1(-th, b, -1, 0, 0);
        em.cx(a, b);
        em.h(b);
        const double dl[3] = {-1, 0, 0};
        em.u2(-kPi, kPi - th, a, kZero3, dl);
        break;
    }
    case RZZ:                                                           // :1288-1294
        em.cx(q[0], q[1]); em.u1(th, q[1], 1, 0, 0); em.cx(q[0], q[1]);
        break;
    case RCCX: {                                                        // :1298-1310
        const uint32_t a = q[0], b = q[1], c = q[2];
        em.u2(0, kPi, c, kZero3, kZero3); em.u1(kPi / 4, c); em.cx(b, c); em.u1(-kPi / 4, c);
        em.cx(a, c); em.u1(kPi / 4, c); em.cx(b, c); em.u1(-kPi / 4, c);
        em.u2(0, kPi, c, kZero3, kZero3);
        break;
    }
    case RC3X: {                                                        // :1314-1335
        const uint32_t a = q[0], b = q[1], c = q[2], d = q[3];
        em.u2(0, kPi, d, kZero3, kZero3); em.u1(kPi / 4, d); em.cx(c, d); em.u1(-kPi / 4, d);
        em.u2(0, kPi, d, kZero3, kZero3); em.cx(a, d); em.u1(kPi / 4, d); em.cx(b, d);
        em.u1(-kPi / 4, d); em.cx(a, d); em.u1(kPi / 4, d); em.cx(b, d);
        em.u1(-kPi / 4, d); em.u2(0, kPi, d, kZero3, kZero3); em.u1(kPi / 4, d); em.cx(c, d);
        em.u1(-kPi / 4, d); em.u2(0, kPi, d, kZero3, kZero3);
        break;
    }
    case C3X: em.c3x_like(kPi / 4, q[0], q[1], q[2], q[3]); break;
    case C3SQRTX: em.c3x_like(kPi / 8, q[0], q[1], q[2], q[3]); break;
    case C4X: {                                                         // :1408-1420
        const uint32_t a = q[0], b = q[1], c = q[2], d = q[3], e = q[4];
        em.h(e); em.cu1(-kPi / 2, d, e); em.h(e);
        em.c3x_like(kPi / 4, a, b, c, d);
        em.h(d); em.cu1(kPi / 4, d, e); em.h(d);
        em.c3x_like(kPi / 4, a, b, c, d);
        em.c3x_like(kPi / 8, a, b, c, e);
        break;
    }
    case R: {                                                           // :924-933
        EOp& e = em.push(F_R, q[0]);
        e.m[0] = th;
        e.kind = EK_R;
        e.ang[0] = th;
        e.jac[0][0] = 1;
        break;
    }
    case SRN: em.fixed(F_SRN, q[0]); break;
    case W:   em.fixed(F_W, q[0]); break;
    case RYY: {                                                         // :1444-1454
        const uint32_t a = q[0], b = q[1];
        em.rx(kPi / 2, a); em.rx(kPi / 2, b); em.cx(a, b);
        em.u1(th, b, 1, 0, 0);                                           // RZ(theta) = U1
        em.cx(a, b); em.rx(-kPi / 2, a); em.rx(-kPi / 2, b);
        break;
    }
    default:
        return false;
    }
    return true;
}

double reference_sweeps(uint32_t op)
{
    // Elementary sweeps of the reference GPU path; a Z/S/SDG/T/TDG/R/CX sweep only
    // touches half of the amplitudes and counts 1/2 (per-gate algorithmic model).
    static std::vector<double> table;
    if (table.empty()) {
        table.resize(N_REF_OPS);
        for (uint32_t o = 0; o < N_REF_OPS; o++) {
            std::vector<EOp> ops;
            svb_gate g{};
            g.op = o;
            for (int i = 0; i < 5; i++) g.qb[i] = i;
            lower_gate(g, 0, ops);
            double s = 0;
            for (const EOp& e : ops)
                s += (e.form == F_CX || (form_is_diag(e.form) && e.form != F_U1)) ? 0.5 : 1.0;
            table[o] = s;
        }
    }
    return op < table.size() ? table[op] : 0.0;
}

}  // namespace svb
