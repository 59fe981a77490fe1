// Per-amplitude-pair arithmetic of the elementary forms, shared by every engine.
// Each case writes the same expression as the reference gate body it names
// (svsim/src/svsim_nvgpu_sin.cuh), evaluated in the state's precision.
#pragma once

#include <cuda_runtime.h>
#include <type_traits>

#include "svb_internal.h"

#define SVB_HD __host__ __device__ __forceinline__

namespace svb {

template <typename T> struct VecOf;
template <> struct VecOf<double> { using type = double2; };
template <> struct VecOf<float> { using type = float2; };

template <typename T>
struct Coef {               // the op's 8 parameters in the state's precision
    T m[8];
};

template <typename T>
SVB_HD Coef<T> load_coef(const double* m)
{
    Coef<T> c;
#pragma unroll
    for (int i = 0; i < 8; i++) c.m[i] = static_cast<T>(m[i]);
    return c;
}

// Dense forms: (a0, a1) -> (b0, b1).  `form` is uniform across the warp.
template <typename T, typename V>
SVB_HD void dense_pair(int form, const Coef<T>& c, V& a0, V& a1)
{
    const T a0r = a0.x, a0i = a0.y, a1r = a1.x, a1i = a1.y;
    const T S2I = static_cast<T>(0.70710678118654752440);
    switch (form) {
    case F_C1:   // C1_GATE :654-675
        a0.x = (c.m[0] * a0r) - (c.m[1] * a0i) + (c.m[2] * a1r) - (c.m[3] * a1i);
        a0.y = (c.m[0] * a0i) + (c.m[1] * a0r) + (c.m[2] * a1i) + (c.m[3] * a1r);
        a1.x = (c.m[4] * a0r) - (c.m[5] * a0i) + (c.m[6] * a1r) - (c.m[7] * a1i);
        a1.y = (c.m[4] * a0i) + (c.m[5] * a0r) + (c.m[6] * a1i) + (c.m[7] * a1r);
        break;
    case F_X:    // X_GATE :818-830
        a0.x = a1r; a0.y = a1i; a1.x = a0r; a1.y = a0i;
        break;
    case F_Y:    // Y_GATE :837-850
        a0.x = a1i; a0.y = -a1r; a1.x = -a0i; a1.y = a0r;
        break;
    case F_H:    // H_GATE :873-887
        a0.x = S2I * (a0r + a1r); a0.y = S2I * (a0i + a1i);
        a1.x = S2I * (a0r - a1r); a1.y = S2I * (a0i - a1i);
        break;
    case F_SRN:  // SRN_GATE :894-907
        a0.x = T(0.5) * (a0r + a1r); a0.y = T(0.5) * (a0i - a1i);
        a1.x = T(0.5) * (a0r + a1r); a1.y = T(0.5) * (-a0i + a1i);
        break;
    case F_W:    // W_GATE :1428-1440
        a0.x = S2I * (a0r + a1i); a0.y = S2I * (a0i - a1r);
        a1.x = S2I * (a0i + a1r); a1.y = S2I * (-a0r + a1i);
        break;
    case F_RX:   // RX_GATE :1085-1100
        a0.x = (c.m[0] * a0r) - (c.m[1] * a1i);
        a0.y = (c.m[0] * a0i) + (c.m[1] * a1r);
        a1.x = -(c.m[1] * a0i) + (c.m[0] * a1r);
        a1.y = +(c.m[1] * a0r) + (c.m[0] * a1i);
        break;
    case F_RY:   // RY_GATE :1104-1122
        a0.x = (c.m[0] * a0r) + (c.m[1] * a1r);
        a0.y = (c.m[0] * a0i) + (c.m[1] * a1i);
        a1.x = (c.m[2] * a0r) + (c.m[3] * a1r);
        a1.y = (c.m[2] * a0i) + (c.m[3] * a1i);
        break;
    default:
        break;
    }
}

// Diagonal forms act on the |1> amplitude only (F_DIAG also scales |0>: see diag0).
template <typename T, typename V>
SVB_HD void diag_one(int form, const Coef<T>& c, V& a1)
{
    const T a1r = a1.x, a1i = a1.y;
    const T S2I = static_cast<T>(0.70710678118654752440);
    switch (form) {
    case F_Z:   a1.x = -a1r; a1.y = -a1i; break;                               // :857-866
    case F_S:   a1.x = -a1i; a1.y = a1r; break;                                // :940-948
    case F_SDG: a1.x = a1i;  a1.y = -a1r; break;                               // :955-963
    case F_T:   a1.x = S2I * (a1r - a1i); a1.y = S2I * (a1r + a1i); break;     // :970-978
    case F_TDG: a1.x = S2I * (a1r + a1i); a1.y = S2I * (-a1r + a1i); break;    // :985-993
    case F_R:   a1.x = -(a1i * c.m[0]); a1.y = a1r * c.m[0]; break;            // :924-933
    case F_U1:                                                                 // :1022-1038
        a1.x = (c.m[0] * a1r) - (c.m[1] * a1i);
        a1.y = (c.m[0] * a1i) + (c.m[1] * a1r);
        break;
    case F_DIAG:
        a1.x = (c.m[2] * a1r) - (c.m[3] * a1i);
        a1.y = (c.m[2] * a1i) + (c.m[3] * a1r);
        break;
    default:
        break;
    }
}

// |0> side of F_DIAG (identity for every reference form).
template <typename T, typename V>
SVB_HD void diag_zero(int form, const Coef<T>& c, V& a0)
{
    if (form == F_DIAG) {
        const T r = a0.x, i = a0.y;
        a0.x = (c.m[0] * r) - (c.m[1] * i);
        a0.y = (c.m[0] * i) + (c.m[1] * r);
    }
}

// Insert a zero bit at position `b` of `x`.
SVB_HD uint64_t insert_zero(uint64_t x, int b)
{
    const uint64_t lo = x & ((1ull << b) - 1);
    return ((x >> b) << (b + 1)) | lo;
}

}  // namespace svb
