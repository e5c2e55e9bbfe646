// Separable blend functions B(s, d) and their partials, device side.
//
// Same piecewise definitions as the reference (blend_mode.hpp:88-196,
// including the 1e-5 branch cuts of Dodge/Burn and the SoftLight curve),
// evaluated in the solver's arithmetic type. The mode is warp-uniform (it
// comes from the layer descriptor), so the switch never diverges; the
// branches inside a mode are data-dependent selects.
#pragma once
#include <cuda_runtime.h>

namespace unb {

template <class T> __device__ __forceinline__ T dsqrt(T v);
template <> __device__ __forceinline__ float dsqrt<float>(float v) { return sqrtf(v); }
template <> __device__ __forceinline__ double dsqrt<double>(double v) { return sqrt(v); }

template <class T> __device__ __forceinline__ T softlight_g(T d) {
    return d <= T(0.25) ? ((T(16) * d - T(12)) * d + T(4)) * d : dsqrt(d);
}

// Value B(s,d).
template <class T> __device__ __forceinline__ T blend_value(int mode, T s, T d) {
    const T one = T(1), two = T(2), eps = T(1e-5);
    switch (mode) {
    case 0: return s;
    case 1: return s * d;
    case 2: return one - (one - s) * (one - d);
    case 3: return d <= T(0.5) ? two * s * d : one - two * (one - s) * (one - d);
    case 4: return s < d ? s : d;
    case 5: return s < d ? d : s;
    case 6: {
        if (d < eps) return T(0);
        const T q = one - s;
        if (q < eps) return one;
        const T v = d / q;
        return v < one ? v : one;
    }
    case 7: {
        if (one - d < eps) return one;
        if (s < eps) return T(0);
        const T v = (one - d) / s;
        return one - (v < one ? v : one);
    }
    case 8: return s <= T(0.5) ? two * s * d : one - two * (one - s) * (one - d);
    case 9:
        if (s <= T(0.5)) return d - (one - two * s) * d * (one - d);
        return d + (two * s - one) * (softlight_g(d) - d);
    case 10: return s < d ? d - s : s - d;
    case 11: return s + d - two * s * d;
    case 12: return s + d;
    default: return T(0);
    }
}

// Value and both partials at once (the adjoint sweep needs all three).
template <class T> __device__ __forceinline__ void blend_all(int mode, T s, T d, T& f, T& fs, T& fd) {
    const T one = T(1), two = T(2), eps = T(1e-5);
    switch (mode) {
    case 0: f = s; fs = one; fd = T(0); return;
    case 1: f = s * d; fs = d; fd = s; return;
    case 2: f = one - (one - s) * (one - d); fs = one - d; fd = one - s; return;
    case 3:
        if (d <= T(0.5)) { f = two * s * d; fs = two * d; fd = two * s; }
        else { f = one - two * (one - s) * (one - d); fs = two * (one - d); fd = two * (one - s); }
        return;
    case 4: if (s < d) { f = s; fs = one; fd = T(0); } else { f = d; fs = T(0); fd = one; } return;
    case 5: if (s < d) { f = d; fs = T(0); fd = one; } else { f = s; fs = one; fd = T(0); } return;
    case 6: {
        if (d < eps) { f = T(0); fs = T(0); fd = T(0); return; }
        const T q = one - s;
        if (q < eps) { f = one; fs = T(0); fd = T(0); return; }
        const T v = d / q;
        if (one < v) { f = one; fs = T(0); fd = T(0); return; }
        f = v; fs = d / (q * q); fd = one / q;
        return;
    }
    case 7: {
        if (one - d < eps) { f = one; fs = T(0); fd = T(0); return; }
        if (s < eps) { f = T(0); fs = T(0); fd = T(0); return; }
        const T v = (one - d) / s;
        if (one < v) { f = T(0); fs = T(0); fd = T(0); return; }
        f = one - v; fs = (one - d) / (s * s); fd = one / s;
        return;
    }
    case 8:
        if (s <= T(0.5)) { f = two * s * d; fs = two * d; fd = two * s; }
        else { f = one - two * (one - s) * (one - d); fs = two * (one - d); fd = two * (one - s); }
        return;
    case 9:
        if (s <= T(0.5)) {
            f = d - (one - two * s) * d * (one - d);
            fs = two * d * (one - d);
            fd = two * s + two * d - T(4) * s * d;
        } else {
            const bool low = d <= T(0.25);
            const T g = low ? ((T(16) * d - T(12)) * d + T(4)) * d : dsqrt(d);
            const T h = low ? (T(48) * d * d - T(24) * d + T(4)) : (one / (two * dsqrt(d)));
            f = d + (two * s - one) * (g - d);
            fs = two * (g - d);
            fd = one + (two * s - one) * h - (two * s - one);
        }
        return;
    case 10: if (s < d) { f = d - s; fs = -one; fd = one; } else { f = s - d; fs = one; fd = -one; } return;
    case 11: f = s + d - two * s * d; fs = one - two * d; fd = one - two * s; return;
    case 12: f = s + d; fs = one; fd = one; return;
    default: f = T(0); fs = T(0); fd = T(0); return;
    }
}

// Quotient: the FP32 solver uses the fast reciprocal-based division (its
// results carry FP32 rounding anyway); FP64 keeps IEEE division.
template <class T> __device__ __forceinline__ T qdiv(T a, T b);
template <> __device__ __forceinline__ float qdiv<float>(float a, float b) { return __fdividef(a, b); }
template <> __device__ __forceinline__ double qdiv<double>(double a, double b) { return a / b; }

template <class T>
__device__ __noinline__ void blend_special(int sp, T s, T d, T& f, T& fs, T& fd, bool partials);

// Table-driven blend for the FP32 solver: the ten piecewise-bilinear modes
// without any jump (coefficients selected by a compare); Dodge, Burn and
// SoftLight (a layer-uniform branch) in one out-of-line function, so that
// their code is not copied into every unrolled layer of the solver. Same
// piecewise definitions as blend_all.
template <class T, class M>
__device__ __forceinline__ void blend_table(const M& m, int l, T s, T d, T& f, T& fs, T& fd, bool partials) {
    const int sp = m.special[l];
    if (sp == 0) {
        const T t = m.ka[l] * s + m.kb[l] * d + m.kc[l];
        const bool c = m.strict[l] ? (t < T(0)) : (t <= T(0));
        const T c0 = c ? m.c0[l][0] : m.c0[l][1];
        const T cs = c ? m.cs[l][0] : m.cs[l][1];
        const T cd = c ? m.cd[l][0] : m.cd[l][1];
        const T csd = c ? m.csd[l][0] : m.csd[l][1];
        f = __fmaf_rn(csd * s, d, __fmaf_rn(cd, d, __fmaf_rn(cs, s, c0)));
        if (partials) { fs = __fmaf_rn(csd, d, cs); fd = __fmaf_rn(csd, s, cd); }
        return;
    }
    blend_special<T>(sp, s, d, f, fs, fd, partials);
}

template <class T>
__device__ __noinline__ void blend_special(int sp, T s, T d, T& f, T& fs, T& fd, bool partials) {
    const T one = T(1), two = T(2), eps = T(1e-5);
    if (sp == 6) {
        const T q = one - s;
        const T v = qdiv(d, q);
        const bool flat = d < eps || q < eps || one < v;
        f = d < eps ? T(0) : (q < eps ? one : (v < one ? v : one));
        if (partials) { fs = flat ? T(0) : qdiv(v, q); fd = flat ? T(0) : qdiv(one, q); }
    } else if (sp == 7) {
        const T v = qdiv(one - d, s);
        const bool flat = one - d < eps || s < eps || one < v;
        f = one - d < eps ? one : (s < eps ? T(0) : one - (v < one ? v : one));
        if (partials) { fs = flat ? T(0) : qdiv(v, s); fd = flat ? T(0) : qdiv(one, s); }
    } else {
        const bool low = d <= T(0.25);
        const T r = dsqrt(d);
        const T g = low ? ((T(16) * d - T(12)) * d + T(4)) * d : r;
        if (s <= T(0.5)) {
            f = d - (one - two * s) * d * (one - d);
            if (partials) { fs = two * d * (one - d); fd = two * s + two * d - T(4) * s * d; }
        } else {
            f = d + (two * s - one) * (g - d);
            if (partials) {
                const T h = low ? (T(48) * d * d - T(24) * d + T(4)) : qdiv(one, two * r);
                fs = two * (g - d);
                fd = one + (two * s - one) * h - (two * s - one);
            }
        }
    }
}

}  // namespace unb
