// nnp_math.cuh -- FP32 device versions of the reference's basis functions,
// cutoffs and activations.  Each follows the cited reference formula; where
// the reference formula overflows in FP32 (it is written for FP64) the same
// function is evaluated in an algebraically equal, overflow-free form, which
// the comment says.  Transcendentals are CUDA's own expf/tanhf/... .
#pragma once

#include <cuda_runtime.h>

#include "nnp_internal.h"

namespace nnp {

#define NNP_PI_F 3.14159265358979f
#define NNP_RAD2_F 1.41421356237310f
#define NNP_RADPI_F 1.77245385090552f
#define NNP_LOG2_F 0.69314718055995f

// Cutoff::cutf / cutg (src/nnp/cutoff.cpp:62-114).  COS uses sincospif, the
// reference a degree-15/16 Taylor series of cos/sin about pi/2 whose error
// (<1e-11) is far below FP32 resolution.
__device__ __forceinline__ void cutoff_fg(const DevCut &c, float r, float &f, float &g)
{
    f = 0.f;
    g = 0.f;
    if (!(r < c.rc)) return;
    switch (c.name) {
    case CUT_STEP: f = 1.f; break;
    case CUT_COS: {
        float s, co;
        sincospif(r * c.rci, &s, &co);
        f = 0.5f * (co + 1.f);
        g = -0.5f * c.pirci * s;
    } break;
    case CUT_TANH: {
        const float t = tanhf(1.f - r * c.rci);
        f = t * t * t;
        g = -3.f * t * t * (1.f - t * t) * c.rci;
    } break;
    case CUT_POLY3: {
        const float x = r * c.rci;
        f = (2.f * x - 3.f) * x * x + 1.f;
        g = 6.f * x * (x - 1.f) * c.rci;
    } break;
    default: break;
    }
}

// sech(x) and tanh(x) from e = exp(-|x|) (no overflow for any x)
__device__ __forceinline__ void sech_tanh(float x, float &s, float &t)
{
    const float e = expf(-fabsf(x));
    const float e2 = e * e;
    const float den = 1.f / (1.f + e2);
    s = 2.f * e * den;
    t = copysignf((1.f - e2) * den, x);
}

// BasisR::symmf / symmd (src/nnp/basis_radial.cpp:175-257): value G(r) and
// derivative dG/dr of one radial function with cutoff value fc and slope fcd.
__device__ __forceinline__ void radial_fd(int form, float r, float rs, float eta, float fc, float fcd,
                                          float &val, float &der)
{
    switch (form) {
    case RAD_GAUSSIAN: {
        const float arg = eta * (r - rs);
        const float e = expf(-arg * arg);
        val = e * fc;
        der = e * (-2.f * eta * arg * fc + fcd);
    } break;
    case RAD_SECH: {            // 2e/(1+e^2) with e=exp(-x) is sech(x)
        float s, t;
        sech_tanh(eta * (r - rs), s, t);
        val = s * fc;
        der = s * (-eta * t * fc + fcd);
    } break;
    case RAD_LOGISTIC: {        // 4e/(1+e)^2 with e=exp(-2x) is sech(x)^2
        float s, t;
        sech_tanh(eta * (r - rs), s, t);
        val = s * s * fc;
        der = s * s * (-2.f * eta * t * fc + fcd);
    } break;
    case RAD_TANH: {
        const float t = tanhf(-eta * (r - rs));
        val = 0.5f * (t + 1.f) * fc;
        der = 0.5f * (-eta * (1.f - t * t) * fc + (1.f + t) * fcd);
    } break;
    case RAD_LOGCOSH: {         // 0.5*log1p(exp(y)), y=-2x, as a stable softplus
        const float y = -2.f * eta * (r - rs);
        const float sp = (y > 0.f) ? y + log1pf(expf(-y)) : log1pf(expf(y));
        const float sg = 1.f / (1.f + expf(-y));          // e/(1+e)
        val = 0.5f * sp * fc;
        der = -eta * sg * fc + 0.5f * sp * fcd;
    } break;
    case RAD_LOGCOSH2: {        // a*e/(e-1) = a/(1-q), e=exp(k a), q=exp(-k a), k=2*sqrt(2)
        const float k = 2.f * NNP_RAD2_F;
        const float a = -eta * (r - rs);
        float f, fa;            // f(a) and df/da
        if (fabsf(a) < 1e-3f) {
            f = 1.f / k + 0.5f * a + k * a * a / 12.f;
            fa = 0.5f + k * a / 6.f;
        } else {
            const float q = expf(-k * a);
            const float om = -expm1f(-k * a);              // 1-q
            f = a / om;
            fa = (om - k * a * q) / (om * om);
        }
        val = f * fc;
        der = fa * (-eta) * fc + f * fcd;
    } break;
    default: val = 0.f; der = 0.f;
    }
}

// x^n for a small non-negative integer n by binary powering (exact products,
// the same value pow(x, double(n)) rounds to within an ulp or two)
__device__ __forceinline__ float ipow(float x, int n)
{
    float r = 1.f;
    while (n) {
        if (n & 1) r *= x;
        x *= x;
        n >>= 1;
    }
    return r;
}

__device__ __forceinline__ float zpow(float x, float zeta, int izeta)
{
    if (izeta >= 0) return ipow(x, izeta);
    return (x > 0.f) ? exp2f(zeta * log2f(x)) : ((zeta == 0.f) ? 1.f : 0.f);
}

// Angular functions other than GAUSS (BasisA::symmf / symmd,
// basis_angular.cpp:212-364) for one function: value h and the partials
// dh/dcos, dh/drj, dh/drk.  cj,ck are cutoff values, gj,gk their slopes.
__device__ __forceinline__ void angular_generic(int form, float rj, float rk, float cs, float cj, float ck,
                                                float gj, float gk, float lf, float zeta, int izeta,
                                                float ieta2, bool want_der, float &h, float &hc,
                                                float &hrj, float &hrk)
{
    const float r2s = rj * rj + rk * rk;
    const float cw = fabsf(0.5f + lf * cs);
    const float pm1 = zpow(cw, zeta - 1.f, izeta > 0 ? izeta - 1 : -1);
    const float pz = (izeta == 0) ? 1.f : pm1 * cw;
    float rad, dfac;            // radial factor and d(rad)/dr_j = -2 r_j * dfac * rad
    switch (form) {
    case ANG_GAUSS: {
        rad = expf(-ieta2 * r2s);
        dfac = ieta2;
    } break;
    case ANG_GAUSS2: {
        const float fd = expf(-0.5f * NNP_PI_F * ieta2 * r2s);
        const float den = 1.f / (1.f + fd);
        rad = 2.f * fd * den;
        dfac = 0.5f * NNP_PI_F * ieta2 * den;
    } break;
    case ANG_SECH: {
        const float fd = expf(-0.5f * NNP_PI_F * ieta2 * r2s);
        const float fd2 = fd * fd, den = 1.f / (1.f + fd2);
        rad = 2.f * fd * den;
        dfac = 0.5f * NNP_PI_F * ieta2 * (1.f - fd2) * den;
    } break;
    case ANG_STUDENT3: case ANG_STUDENT4: case ANG_STUDENT5: {
        const int p = 4 + (form - ANG_STUDENT3);
        const float den = rsqrtf(1.f + ieta2 * r2s);
        rad = ipow(den, p);
        dfac = ieta2 * 0.5f * (float)p * den * den;
    } break;
    default: rad = 0.f; dfac = 0.f;
    }
    h = pz * rad * cj * ck;
    if (want_der) {
        hc = zeta * lf * pm1 * rad * cj * ck;
        hrj = pz * rad * (-2.f * rj * cj * dfac + gj) * ck;
        hrk = pz * rad * (-2.f * rk * ck * dfac + gk) * cj;
    }
}

// AFFPBP activations (src/ml/nn.cpp:148-848): a = f(z), d = f'(z); with
// want_d2 also f''(z) (AFFPBP2) for the activations the training path supports.
__device__ __forceinline__ void activation(int neuron, float c, float z, float &a, float &d, float &d2)
{
    d2 = 0.f;
    switch (neuron) {
    case NEU_LINEAR: a = z; d = 1.f; break;
    case NEU_SIGMOID: {
        const float e = expf(-c * fabsf(z));
        const float fr = 1.f / (1.f + e);
        a = (z >= 0.f) ? fr : e * fr;
        d = c * e * fr * fr;
        d2 = (z >= 0.f) ? -c * c * e * (1.f - e) * fr * fr * fr : -c * c * e * (e - 1.f) * fr * fr * fr;
    } break;
    case NEU_TANH: {
        const float t = tanhf(c * z);
        a = t;
        d = c * (1.f - t * t);
        d2 = c * c * (-2.f * t * (1.f - t * t));
    } break;
    case NEU_ISRU: {
        const float zz = c * z, isr = rsqrtf(1.f + zz * zz);
        a = zz * isr;
        d = c * isr * isr * isr;
    } break;
    case NEU_ARCTAN: {
        const float zz = c * z * NNP_PI_F / 2.f;
        a = (2.f / NNP_PI_F) * atanf(zz);
        d = c / (1.f + zz * zz);
    } break;
    case NEU_RELU: a = (z > 0.f) ? z : 0.f; d = (z > 0.f) ? 1.f : 0.f; break;
    case NEU_ELU:
        if (z >= 0.f) { a = z; d = 1.f; } else { const float e = expf(c * z); a = e - 1.f; d = c * e; }
        break;
    case NEU_TANHRE:
        if (z >= 0.f) { a = z; d = 1.f; } else { const float e = expf(2.f * c * z); a = (e - 1.f) / (e + 1.f); d = c * (1.f - a * a); }
        break;
    case NEU_SQRE:
        if (z >= 0.f) { a = z; d = 1.f; } else { const float den = rsqrtf(1.f + z * z); a = z * den; d = den * den * den; }
        break;
    case NEU_SWISH: {
        const float zz = c * z;
        if (zz > 0.f) { const float e = expf(-zz), den = 1.f / (1.f + e); a = z * den; d = (1.f + e * (1.f + zz)) * den * den; }
        else { const float e = expf(zz), den = 1.f / (1.f + e); a = z * e * den; d = e * (1.f + zz + e) * den * den; }
    } break;
    case NEU_GELU: {
        const float zz = 0.5f * NNP_RADPI_F * c * z, ep1 = 1.f + erff(zz);
        a = 0.5f * z * ep1;
        d = 0.5f * (ep1 + c * z * expf(-zz * zz));
    } break;
    case NEU_MISH: {
        const float zz = c * z;
        if (zz > 0.f) {
            const float e = expf(-zz), e2 = e * e, den = 1.f / ((1.f + e) * (1.f + e) + e2);
            a = z * (1.f - 2.f * e2 * den);
            d = 1.f - 2.f * e2 * den * (1.f - 2.f * zz * (1.f + e) * den);
        } else {
            const float e = expf(zz), den = 1.f / (e * (e + 2.f) + 2.f);
            a = z * e * (e + 2.f) * den;
            d = 1.f + 2.f * den * (-1.f + 2.f * zz * (1.f - (e + 2.f) * den));
        }
    } break;
    case NEU_PFLU: {
        const float zz = c * z, z2 = zz * zz, fs = rsqrtf(z2 + 1.f);
        a = 0.5f * z * (1.f + zz * fs);
        d = 0.5f * (zz * (z2 + 2.f) * fs * fs * fs + 1.f);
    } break;
    case NEU_LOGISH: {
        const float l2i = 1.f / NNP_LOG2_F, e = expf(-z), lf = logf(1.f + 1.f / (1.f + e));
        a = l2i * z * lf;
        d = l2i * (lf + z * e / ((1.f + e) * (2.f + e)));
    } break;
    case NEU_SOFTPLUS: {
        const float ci = 1.f / c;
        if (z > 0.f) { const float e = expf(-c * z); a = z + ci * (log1pf(e) - NNP_LOG2_F); d = 1.f / (e + 1.f); }
        else { const float e = expf(c * z); a = ci * (log1pf(e) - NNP_LOG2_F); d = e / (e + 1.f); }
    } break;
    case NEU_SQPLUS: {
        const float ci = 1.f / c, zz = c * z, fs = sqrtf(1.f + zz * zz);
        a = 0.5f * ci * (zz - 1.f + fs);
        d = 0.5f * (zz / fs + 1.f);
    } break;
    case NEU_ATISH: {
        const float zz = 0.5f * NNP_PI_F * z;
        a = z * 0.5f * (1.f + 2.f / NNP_PI_F * atanf(zz));
        d = 0.5f * (1.f + z / (1.f + zz * zz)) + 1.f / NNP_PI_F * atanf(zz);
    } break;
    case NEU_IERF: {            // reference uses the A&S 7.1.26 erf approximation
        const float fexp = expf(-z * z);
        const float zs = (float)((0.f < z) - (z < 0.f));
        const float t = 1.f / (1.f + 0.3275911f * z * zs);
        const float ferf = zs * (1.f - t * (0.254829592f + t * (-0.284496736f + t * (1.421413741f + t * (-1.453152027f + t * 1.061405429f)))) * fexp);
        a = 0.5f * (z * ferf + (fexp + z * NNP_RADPI_F - 1.f) / NNP_RADPI_F);
        d = 0.5f * (ferf + 1.f);
    } break;
    case NEU_TEST: {
        const float zz = c * z, z2 = zz * zz, z4 = z2 * z2, den = rsqrtf(sqrtf(z4 + 1.f));
        a = 0.5f * z * (1.f + zz * den);
        d = 0.5f * (zz * den * (1.f + 1.f / (z4 + 1.f)) + 1.f);
    } break;
    default: a = 0.f; d = 0.f;
    }
}

}  // namespace nnp
