// nnp_device.cuh -- device-side types and building blocks of the NNP path.
//
// Shared by the prebuilt kernels (nnp_kernels.cu, nvcc) and the kernels that
// nnp_jit.cpp specialises at run time for one potential (NVRTC), so it uses
// plain CUDA C++ only: no host headers, no standard library.
//
// Basis functions, cutoffs and activations are FP32 versions of the cited
// reference formulas; where a reference formula overflows in FP32 (it is
// written for FP64) the same function is evaluated in an algebraically equal,
// overflow-free form, which the comment says.  Transcendentals are CUDA's own
// expf/tanhf/... .
#pragma once

#define NNP_MAX_TYPES 8
#define NNP_MAX_TT (NNP_MAX_TYPES * (NNP_MAX_TYPES + 1) / 2)
#define NNP_MAX_LAYERS 8
#define NNP_MAX_RFUNC 32      // radial functions in one (centre, neighbour) block
#define NNP_MAX_AFUNC 32      // angular functions in one (centre, pair) block
#define NNP_MAX_DAMP 8        // distinct GAUSS damping factors per centre type
#define NNP_MAX_CUT 4         // distinct (cutoff form, rc) pairs in a potential
#define NNP_MAX_NODES 128     // widest network layer handled on the device
#define NNP_MAX_NBR 256       // neighbours per atom staged in shared memory
#define NNP_MAX_IMAGES 64     // cell images searched on each side in one lattice direction

#define NNP_WARPS 8           // warps per block of the per-atom kernels
#define NNP_SYMM_CHUNK 8      // angular functions accumulated in registers per pass
#define NNP_PCH 288           // default pair coefficients of one force-kernel chunk
#ifndef NNP_FORCE_CHUNK
#define NNP_FORCE_CHUNK NNP_PCH   // pair coefficients of one chunk of this build's force kernel (<= NNP_PCH)
#endif
#define NNP_FULL 0xffffffffu

#ifdef __CUDACC__
#define NNP_HD __host__ __device__
#else
#define NNP_HD
#endif

namespace nnp {

typedef long long i64;

// Row stride of a transposed weight matrix W^T (ni x no) in shared memory:
// odd, so lanes reading a column (fixed n, consecutive m) hit distinct banks.
NNP_HD inline int wt_stride(int no) { return (no % 2 == 0) ? no + 1 : no + 2; }

// Cutoff::Name, BasisR::Name, BasisA::Name, NN::Neuron numbering of the reference
enum CutName { CUT_NONE = 0, CUT_STEP, CUT_COS, CUT_TANH, CUT_POLY3 };
enum RadName { RAD_NONE = 0, RAD_GAUSSIAN, RAD_SECH, RAD_LOGISTIC, RAD_TANH, RAD_LOGCOSH, RAD_LOGCOSH2 };
enum AngName { ANG_NONE = 0, ANG_GAUSS, ANG_GAUSS2, ANG_SECH, ANG_STUDENT3, ANG_STUDENT4, ANG_STUDENT5 };
enum Neuron {
    NEU_NONE = 0, NEU_LINEAR, NEU_SIGMOID, NEU_TANH, NEU_ISRU, NEU_ARCTAN, NEU_RELU, NEU_ELU, NEU_TANHRE,
    NEU_SQRE, NEU_SWISH, NEU_GELU, NEU_MISH, NEU_PFLU, NEU_LOGISH, NEU_SOFTPLUS, NEU_SQPLUS, NEU_ATISH,
    NEU_IERF, NEU_TEST
};

// ---------------------------------------------------------------- device model
struct DevCut { int name; float rc, rci, pirci; };

struct DevBlockR {
    int n;        // functions
    int off_g;    // offset of the block inside G
    int form;     // RadName
    int cut;      // index into DevPot::cut
    int par;      // first function in rpar (float2: rs, eta)
};

struct DevBlockA {
    int n;
    int off_g;    // absolute offset in G (nInputR + offsetA)
    int form;     // AngName
    int cut;
    int par;      // first function in apar (float4: lambdaf, zeta, ieta2, damp | (izeta+1) << 8)
    int int_zeta; // all zeta are small non-negative integers
};

struct DevType {
    int n_input, n_input_r;
    DevBlockR br[NNP_MAX_TYPES];
    DevBlockA ba[NNP_MAX_TT];
    int ndamp;                      // distinct (cutoff, 1/eta^2) GAUSS damping factors
    float damp_a[NNP_MAX_DAMP];     // 1/eta^2 of the damping factor
    int damp_cut[NNP_MAX_DAMP];     // its cutoff index
    int nlayer;
    int nodes[NNP_MAX_LAYERS + 1];
    int neuron;
    float c;
    i64 woff;                       // first float of this network in wpar
};

struct DevPot {
    int ntypes;
    int ncut;
    float rc;
    double rc_d;
    DevCut cut[NNP_MAX_CUT];
    DevType t[NNP_MAX_TYPES];
};

// device error record: kernels raise flags, the host reads them after a step
struct DevErr {
    int need_cap;     // largest neighbour count seen (when above the capacity)
    int bad_type;     // an atom type was outside [0, ntypes)
    int bad_cell;     // a periodic cell had no volume (1) or was thinner than rc / NNP_MAX_IMAGES (2)
    int nonfinite;    // a non-finite energy or force
};

#if defined(__CUDACC__)

#define NNP_PI_F 3.14159265358979f
#define NNP_RAD2_F 1.41421356237310f
#define NNP_RADPI_F 1.77245385090552f
#define NNP_LOG2_F 0.69314718055995f

// ---------------------------------------------------------------- math

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

// x^n for a small non-negative integer n by binary powering
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

// x^n, 0 <= n < 64, by binary powering with branches on the (warp-uniform) bits of n
__device__ __forceinline__ float upow(float x, int n)
{
    float r = (n & 1) ? x : 1.f;
    if (n >> 1) {
        x *= x;
        if (n & 2) r *= x;
        if (n >> 2) {
            x *= x;
            if (n & 4) r *= x;
            if (n >> 3) {
                x *= x;
                if (n & 8) r *= x;
                if (n >> 4) {
                    x *= x;
                    if (n & 16) r *= x;
                    if (n >> 5) { x *= x; r *= x; }
                }
            }
        }
    }
    return r;
}

// (0.5 + lf cos)^zeta and (.)^(zeta-1), the reference's |0.5 + lambda/2 cos|^zeta
__device__ __forceinline__ void ang_pow(float cs, float lf, float zeta, int iz, float &pz, float &pm1)
{
    const float x = fabsf(fmaf(lf, cs, 0.5f));
    if (iz > 0) {
        pm1 = upow(x, iz - 1);
        pz = pm1 * x;
    } else if (iz == 0) {
        pm1 = 0.f;
        pz = 1.f;
    } else {
        pm1 = (x > 0.f) ? exp2f((zeta - 1.f) * log2f(x)) : 0.f;
        pz = pm1 * x;
    }
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

// AFFPBP activations (src/ml/nn.cpp:148-848): a = f(z), d = f'(z), and
// d2 = f''(z) (AFFPBP2) for the activations the training path uses.
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
    case NEU_IERF: {            // the reference uses the A&S 7.1.26 erf approximation
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

// ---------------------------------------------------------------- warp helpers

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(NNP_FULL, v, o);
    return v;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(NNP_FULL, v, o);
    return v;
}

__device__ __forceinline__ bool finite_d(double x) { return fabs(x) <= 1.7976931348623157e308; }

// accumulate a pair term: FP32 fused multiply-add, or the FP32 product added in FP64
__device__ __forceinline__ void acc_add(float &acc, float a, float b) { acc = fmaf(a, b, acc); }
__device__ __forceinline__ void acc_add(double &acc, float a, float b) { acc += (double)(a * b); }

// ---------------------------------------------------------------- per-atom staging

// Index of damping group d of neighbour k in NbrView::w / wd: the groups are
// stored in pairs, (w_2m, w_2m+1) of a neighbour adjacent, so that one 8-byte
// load reads two groups.
NNP_HD inline int wix(int d, int k, int cap) { return 2 * ((d >> 1) * cap + k) + (d & 1); }

// Per-warp shared-memory view of one atom's neighbours.
struct NbrView {
    float4 *u;          // unit vector to the neighbour and inverse distance (ux, uy, uz, 1/r) [C]
    float *r;           // distance [C]
    float4 *par;        // block parameters [NNP_MAX_AFUNC]
    float4 *raw;        // next atom's neighbour records, prefetched (force views) [C]
    int *j;             // neighbour atom index [C]
    float *fc, *fd;     // cutoff value / slope [ncut][C]
    float *w, *wd;      // GAUSS damping w_e(r) = fc exp(-a_e r^2) and dw_e/dr, groups in pairs (wix)
    float *gx, *gy, *gz;// per-slot gradient dE_i/dd_j [C]
    float *vec;         // dE/dG row of the atom [gstride] (16-byte aligned)
    float *pc;          // pair coefficients [3][pcs]
    int pcs;            // their array length: the chunk, at least one row (C)
    int *seg;           // [NNP_MAX_TYPES+1] type-segment starts
    unsigned char *t;   // neighbour type [C]
};

// length of each pair-coefficient array of a force view: the chunk the
// kernel was built for, and never less than one row (C slots), so that a
// smaller chunk frees shared memory for resident blocks
NNP_HD inline int coef_len(int chunk, int C) { return chunk > C ? chunk : C; }

NNP_HD inline int nbr_view_floats(int C, int ncut, int ndamp, int gstride, bool force, int chunk)
{
    return 4 * C + 4 * NNP_MAX_AFUNC + 2 * C + 2 * ncut * C + 4 * ((ndamp + 1) / 2) * C +
           (force ? 4 * C + 3 * C + gstride + 3 * coef_len(chunk, C) : 0) + NNP_MAX_TYPES + 1 + (C + 3) / 4;
}

__device__ inline NbrView nbr_view(float *base, int C, int ncut, int ndamp, int gstride, bool force)
{
    NbrView v;
    float *p = base;
    v.u = reinterpret_cast<float4 *>(p); p += 4 * C;                 // 16-byte aligned first
    v.par = reinterpret_cast<float4 *>(p); p += 4 * NNP_MAX_AFUNC;
    if (force) {
        v.raw = reinterpret_cast<float4 *>(p); p += 4 * C;           // stays 16-byte aligned
        v.vec = p; p += gstride;                                      // gstride % 4 == 0
    } else {
        v.raw = nullptr;
        v.vec = nullptr;
    }
    v.r = p; p += C;
    v.j = reinterpret_cast<int *>(p); p += C;
    v.fc = p; p += ncut * C;
    v.fd = p; p += ncut * C;
    v.w = p; p += 2 * ((ndamp + 1) / 2) * C;                        // 8-byte aligned (C % 8 == 0)
    v.wd = p; p += 2 * ((ndamp + 1) / 2) * C;
    if (force) {
        v.gx = p; p += C;
        v.gy = p; p += C;
        v.gz = p; p += C;
        v.pcs = coef_len(NNP_FORCE_CHUNK, C);
        v.pc = p; p += 3 * v.pcs;
    } else {
        v.pcs = 0;
        v.gx = v.gy = v.gz = v.pc = nullptr;
    }
    v.seg = reinterpret_cast<int *>(p); p += NNP_MAX_TYPES + 1;
    v.t = reinterpret_cast<unsigned char *>(p);
    return v;
}

// Load an atom's neighbour list into the warp's view and compute the per-neighbour
// quantities: unit vector, distance, cutoff value/slope per cutoff, and the
// GAUSS damping factors w_e(r) = fc(r) exp(-a_e r^2) with slopes dw_e/dr.
// (src: the atom's n neighbour records, in global or shared memory)
__device__ __forceinline__ int stage_records(const NbrView &v, const float4 *src, int n, int cap, const DevPot &P,
                                            const DevType &T, int lane)
{
    for (int k = lane; k < n; k += 32) {
        const float4 e = src[k];
        const float r = sqrtf(e.x * e.x + e.y * e.y + e.z * e.z);
        const float ir = 1.f / r;
        v.u[k] = make_float4(e.x * ir, e.y * ir, e.z * ir, ir);
        v.r[k] = r;
        const int pk = __float_as_int(e.w);
        v.j[k] = pk & 0x0fffffff;
        v.t[k] = (unsigned char)((unsigned)pk >> 28);
        for (int c = 0; c < P.ncut; ++c) {
            float f, g;
            cutoff_fg(P.cut[c], r, f, g);
            v.fc[c * cap + k] = f;
            v.fd[c * cap + k] = g;
        }
        for (int d = 0; d < T.ndamp; ++d) {
            const int c = T.damp_cut[d];
            const float a = T.damp_a[d];
            const float ex = expf(-a * r * r);
            const float f = v.fc[c * cap + k], g = v.fd[c * cap + k];
            v.w[wix(d, k, cap)] = f * ex;
            v.wd[wix(d, k, cap)] = (g - 2.f * a * r * f) * ex;
        }
    }
    // type segment starts (the list is grouped by type)
    for (int t = 0; t <= P.ntypes; ++t) {
        int c = 0;
        for (int kb = 0; kb < n; kb += 32) {
            const int k = kb + lane;
            c += __popc(__ballot_sync(NNP_FULL, k < n && v.t[k] < t));
        }
        if (lane == 0) v.seg[t] = c;
    }
    __syncwarp();
    return n;
}

// Asynchronous copy of n neighbour records (16 bytes each) into shared memory
// (cp.async, completed by async_wait): the next atom's list streams in while
// the warp works on the current one.
__device__ __forceinline__ void prefetch_records(float4 *dst, const float4 *src, int n, int lane)
{
    for (int k = lane; k < n; k += 32) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst + k);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src + k) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// The per-atom kernels walk atoms idx, idx + stride, ... of the element-sorted
// order.  prefetch_atom starts the copy of atom order[idx]'s records (if idx <
// N) and returns its index and count; stage_prefetched waits for them and
// stages them.
__device__ __forceinline__ void prefetch_atom(const NbrView &v, i64 idx, i64 N, const int *__restrict__ order,
                                              const float4 *__restrict__ nbr, const int *__restrict__ nbr_cnt,
                                              int cap, int lane, i64 &i_next, int &n_next)
{
    if (idx < N) {
        i_next = order[idx];
        n_next = nbr_cnt[i_next];
        prefetch_records(v.raw, nbr + i_next * cap, n_next, lane);
    }
}

__device__ __forceinline__ int stage_prefetched(const NbrView &v, int n, int cap, const DevPot &P, const DevType &T,
                                                int lane)
{
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncwarp();
    return stage_records(v, v.raw, n, cap, P, T, lane);
}

// The force kernel's atom walk is a load pipeline: while the warp works on
// one atom, the records of the next stream into shared memory (cp.async),
// then its dE/dG row once the atom's own row is no longer read (during the
// scatter), and the neighbour count and type of the atom after that and the
// index of the third load into registers, so that no global load of the walk
// waits for another.  (A second row buffer would overlap the row with the
// whole atom but costs the shared memory of a resident block at some
// capacities.)  Count and type travel packed: n << 4 | type
// (types at or above 15 read as 15, which no potential has).
__device__ __forceinline__ int pack_nt(int n, int t) { return (n << 4) | (int)min((unsigned)t, 15u); }

// cp.async of n neighbour records into raw and of the first nrow floats of a
// dE/dG row (16-byte chunks; rows are gstride floats, gstride % 4 == 0)
__device__ __forceinline__ void prefetch_rows(float4 *raw, const float4 *src, int n, float *vdst, const float *vsrc,
                                              int nrow, int lane)
{
    for (int k = lane; k < n; k += 32) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(raw + k);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src + k) : "memory");
    }
    for (int k = lane; 4 * k < nrow; k += 32) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(vdst + 4 * k);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(vsrc + 4 * k) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// Lanes of a radial block of n <= 32 functions: G phases per function (the
// largest power of two with G n <= 32), lane = f G + ph; a lane sums the
// neighbours s0 + ph, s0 + ph + G, ... of function f and a shuffle tree over
// the G phases (consecutive lanes) completes the sum.
__device__ __forceinline__ void radial_lanes(int n, int lane, int &f, int &ph, int &G)
{
    G = 1;
    while (4 * G * n <= 64) G <<= 1;        // 2 G n <= 32
    const int lg = __ffs(G) - 1;
    f = lane >> lg;
    ph = lane & (G - 1);
}

// p / m for 0 <= p < 2^22 and 1 <= m <= 1024 without an integer division: the
// approximate float quotient is within one of the exact one, and the two
// comparisons correct it.
__device__ __forceinline__ int small_div(int p, int m)
{
    int q = (int)__fdividef((float)p, (float)m);
    q += ((q + 1) * m <= p) ? 1 : 0;
    q -= (q * m > p) ? 1 : 0;
    return q;
}

// One angular block as seen by a warp: segments of the two neighbour types and
// the numbering of its pairs, p = g*m + f with a fast index f in [0,m):
//  - J != K (rectangle): m = nb, pair (a,b) = (g, f);
//  - J == K (fold):      m = n,  pair (a,b) = (f, (f+g+1) mod n) for
//    g < (n-1)/2, and for even n a last half row g = n/2-1, f < n/2.
//    Every unordered pair of distinct slots appears exactly once:
//    n*floor((n-1)/2) + (n even ? n/2 : 0) = n(n-1)/2 pairs.
// Lanes step p by 32, which is (q32, r32) = (32/m, 32%m) in (g, f): two
// adds and one wrap per step instead of a division or a square root.
// For J != K the larger segment gives the rows (the angular functions are
// symmetric in the two neighbours), so a chunk's row owners and column owners
// fit one pass of the force kernel's slot pass.
// The force kernel stores per-pair coefficients chunk by chunk, a chunk being
// whole rows [g0, g1): pair (g, f) at coefficient index (g - g0) s + f, with
// the row stride s = n (J == K) or nb rounded up to an odd number (J != K),
// so that row owners reading their rows side by side hit distinct banks.
struct Blk {
    int sa, na;       // first member (rows): segment start / size
    int sb, nb;       // second member (columns; sb == sa for J == K)
    bool tri;
    int npairs;
    int m, q32, r32;
    int rows, s;      // rows of pairs (J == K: n/2 with the half row), coefficient row stride
};

__device__ __forceinline__ bool make_blk(const NbrView &v, int J, int K, Blk &k)
{
    const int s0 = v.seg[J], n0 = v.seg[J + 1] - s0;
    k.tri = (J == K);
    if (k.tri) {
        k.sa = k.sb = s0;
        k.na = k.nb = n0;
        k.npairs = n0 * (n0 - 1) / 2;
        k.rows = n0 >> 1;
        k.s = n0;
    } else {
        const int s1 = v.seg[K], n1 = v.seg[K + 1] - s1;
        const bool sw = n1 > n0;
        k.sa = sw ? s1 : s0;
        k.na = sw ? n1 : n0;
        k.sb = sw ? s0 : s1;
        k.nb = sw ? n0 : n1;
        k.npairs = k.na * k.nb;
        k.rows = k.na;
        k.s = k.nb | 1;
    }
    if (k.npairs == 0) return false;
    k.m = k.nb;
    k.q32 = small_div(32, k.m);
    k.r32 = 32 - k.q32 * k.m;
    return true;
}

// rows of one coefficient chunk of the force kernel: as many as NNP_FORCE_CHUNK
// coefficients hold, and for J != K with fewer than 32 columns at most
// 32 - nb, so that rows and columns have one lane each in the slot pass
__device__ __forceinline__ int chunk_rows(const Blk &k)
{
    int R = small_div(NNP_FORCE_CHUNK, k.s);   // R s <= chunk, or R = 1 and s <= cap <= pcs
    if (!k.tri && k.nb < 32) R = min(R, 32 - k.nb);
    return max(R, 1);
}

struct PairIt {
    int f, g;
};

__device__ __forceinline__ PairIt pit_init(const Blk &k, int p)
{
    PairIt it;
    it.g = small_div(p, k.m);
    it.f = p - it.g * k.m;
    return it;
}

__device__ __forceinline__ void pit_next(const Blk &k, PairIt &it)
{
    it.f += k.r32;
    it.g += k.q32;
    if (it.f >= k.m) {
        it.f -= k.m;
        ++it.g;
    }
}

// neighbour slots (a, b) of the pair at `it`
__device__ __forceinline__ void pit_slots(const Blk &k, const PairIt &it, int &a, int &b)
{
    if (k.tri) {
        const int bb = it.f + it.g + 1;
        a = k.sa + it.f;
        b = k.sa + (bb >= k.m ? bb - k.m : bb);
    } else {
        a = k.sa + it.g;
        b = k.sb + it.f;
    }
}

// ---------------------------------------------------------------- generic block code

// Symmetry functions of one angular block, parameters from v.par (any form).
template <typename Acc>
__device__ void symm_block_generic(const NbrView &v, const DevBlockA &B, const Blk &k, int cap, int lane, float *Gi)
{
    if (B.form == ANG_GAUSS) {
        // damping exp(-(ra^2+rb^2)/eta^2) fc(ra) fc(rb) = w(ra) w(rb) from the
        // staged factors; NNP_SYMM_CHUNK functions per pass in registers
        for (int f0 = 0; f0 < B.n; f0 += NNP_SYMM_CHUNK) {
            const int nf = min(NNP_SYMM_CHUNK, B.n - f0);
            Acc acc[NNP_SYMM_CHUNK];
#pragma unroll
            for (int f = 0; f < NNP_SYMM_CHUNK; ++f) acc[f] = 0;
            PairIt it = pit_init(k, lane);
#pragma unroll 1
            for (int p = lane; p < k.npairs; p += 32, pit_next(k, it)) {
                int a, b;
                pit_slots(k, it, a, b);
                const float4 ua = v.u[a], ub = v.u[b];
                const float cs = ua.x * ub.x + ua.y * ub.y + ua.z * ub.z;
                int dcur = -1;
                float damp = 0.f;
#pragma unroll
                for (int f = 0; f < NNP_SYMM_CHUNK; ++f) {
                    if (f < nf) {
                        const float4 q = v.par[f0 + f];
                        const int pk = __float_as_int(q.w);
                        const int d = pk & 0xff, iz = (pk >> 8) - 1;
                        if (d != dcur) {
                            dcur = d;
                            damp = v.w[wix(d, a, cap)] * v.w[wix(d, b, cap)];
                        }
                        float pz, pm1;
                        ang_pow(cs, q.x, q.y, iz, pz, pm1);
                        acc_add(acc[f], pz, damp);
                    }
                }
            }
#pragma unroll
            for (int f = 0; f < NNP_SYMM_CHUNK; ++f) {
                if (f < nf) {
                    const Acc s = warp_sum(acc[f]);
                    if (lane == 0) Gi[B.off_g + f0 + f] = (float)s;
                }
            }
        }
    } else {
        // other forms: one function per pass over the pairs
        for (int f = 0; f < B.n; ++f) {
            const float4 q = v.par[f];
            const int iz = (__float_as_int(q.w) >> 8) - 1;
            Acc acc = 0;
            PairIt it = pit_init(k, lane);
#pragma unroll 1
            for (int p = lane; p < k.npairs; p += 32, pit_next(k, it)) {
                int a, b;
                pit_slots(k, it, a, b);
                const float4 ua = v.u[a], ub = v.u[b];
                const float cs = ua.x * ub.x + ua.y * ub.y + ua.z * ub.z;
                float h, hc, hrj, hrk;
                angular_generic(B.form, v.r[a], v.r[b], cs, v.fc[B.cut * cap + a], v.fc[B.cut * cap + b], 0.f, 0.f, q.x,
                                q.y, iz, q.z, false, h, hc, hrj, hrk);
                acc_add(acc, h, 1.f);
            }
            acc = warp_sum(acc);
            if (lane == 0) Gi[B.off_g + f] = (float)acc;
        }
    }
}

// Writes the three dE/dd coefficients of one pair (see force_body); ira, irb
// are the inverse distances.
__device__ __forceinline__ void pair_coeffs(float *pc, int pcs, int q, float hc, float hra, float hrb, float cs,
                                            float ira, float irb)
{
    pc[q] = hra - hc * cs * ira;                 // on u_a in dE/dd_a
    pc[pcs + q] = hc;                            // on u_b / r_a in dE/dd_a, on u_a / r_b in dE/dd_b
    pc[2 * pcs + q] = hrb - hc * cs * irb;       // on u_b in dE/dd_b
}

// Pair pass of the force kernel for pairs [c0,c1) of one block (any form),
// whole rows, coefficients at it.g s + it.f - qoff, eb = dE/dG of the block:
// dE/dcos, dE/dr_a, dE/dr_b from e = dE/dG of the block's functions.
__device__ inline void force_pairs_generic(const NbrView &v, const DevBlockA &B, const float *eb, const Blk &k, int c0,
                                           int c1, int qoff, int cap, int lane)
{
    const bool gauss = (B.form == ANG_GAUSS);
    PairIt it = pit_init(k, c0 + lane);
#pragma unroll 1
    for (int p = c0 + lane; p < c1; p += 32, pit_next(k, it)) {
        int a, b;
        pit_slots(k, it, a, b);
        const float4 ua = v.u[a], ub = v.u[b];
        const float cs = ua.x * ub.x + ua.y * ub.y + ua.z * ub.z;
        float hc = 0.f, hra = 0.f, hrb = 0.f;
        if (gauss) {
            int dcur = -1;
            float sc = 0.f, sp = 0.f;
            for (int f = 0; f < B.n; ++f) {
                const float4 q = v.par[f];
                const int pk = __float_as_int(q.w);
                const int d = pk & 0xff, iz = (pk >> 8) - 1;
                if (d != dcur) {
                    if (dcur >= 0) {
                        const float wa = v.w[wix(dcur, a, cap)], wb = v.w[wix(dcur, b, cap)];
                        hc = fmaf(sc, wa * wb, hc);
                        hra = fmaf(sp, v.wd[wix(dcur, a, cap)] * wb, hra);
                        hrb = fmaf(sp, wa * v.wd[wix(dcur, b, cap)], hrb);
                    }
                    dcur = d;
                    sc = 0.f;
                    sp = 0.f;
                }
                float pz, pm1;
                ang_pow(cs, q.x, q.y, iz, pz, pm1);
                const float ef = eb[f];
                sc = fmaf(ef * q.y * q.x, pm1, sc);
                sp = fmaf(ef, pz, sp);
            }
            if (dcur >= 0) {
                const float wa = v.w[wix(dcur, a, cap)], wb = v.w[wix(dcur, b, cap)];
                hc = fmaf(sc, wa * wb, hc);
                hra = fmaf(sp, v.wd[wix(dcur, a, cap)] * wb, hra);
                hrb = fmaf(sp, wa * v.wd[wix(dcur, b, cap)], hrb);
            }
        } else {
            const float ca = v.fc[B.cut * cap + a], cb = v.fc[B.cut * cap + b];
            const float ga = v.fd[B.cut * cap + a], gb = v.fd[B.cut * cap + b];
            for (int f = 0; f < B.n; ++f) {
                const float4 q = v.par[f];
                const int iz = (__float_as_int(q.w) >> 8) - 1;
                float h, dc, dra, drb;
                angular_generic(B.form, v.r[a], v.r[b], cs, ca, cb, ga, gb, q.x, q.y, iz, q.z, true, h, dc, dra, drb);
                const float ef = eb[f];
                hc = fmaf(ef, dc, hc);
                hra = fmaf(ef, dra, hra);
                hrb = fmaf(ef, drb, hrb);
            }
        }
        pair_coeffs(v.pc, v.pcs, it.g * k.s + it.f - qoff, hc, hra, hrb, cs, ua.w, ub.w);
    }
}

// Slot pass over the rows [g0, g1) of one chunk: each lane owns neighbour
// slots of the block (for J == K blocks of at most 16 slots, one of the two
// halves of a slot's pairs) and sums, in a fixed order, the coefficients of
// the chunk's pairs that contain them.  With the numbering of Blk, slot x of
// a J == K block is the first member of pair (x, x+g+1 mod n) and the second
// member of pair (x-g-1 mod n, x) in row g; on the half row of an even n only
// first members below n/2 have a pair.

// g += sa u + (1/r) v for the slot with unit vector and 1/r us
__device__ __forceinline__ void slot_add(const NbrView &v, int slot, float4 us, float sa_, float vx, float vy, float vz)
{
    v.gx[slot] += fmaf(sa_, us.x, us.w * vx);
    v.gy[slot] += fmaf(sa_, us.y, us.w * vy);
    v.gz[slot] += fmaf(sa_, us.z, us.w * vz);
}

// J == K: slot x's pairs in rows [g0, g1) in which it is the first (second ==
// false) or the second member; cS is the coefficient on its own unit vector.
// The partner o and the coefficient index (g - g0) n + (first member) advance
// by one row per step.
__device__ __forceinline__ void tri_visits(const NbrView &v, const Blk &k, const float *cS, const float *cH, int x,
                                           bool second, int g0, int g1, float &sa_, float &vx, float &vy, float &vz)
{
    const int n = k.m, hn = n >> 1, hr = (n & 1) ? -1 : hn - 1;   // half row of an even n
    int o = second ? x - g0 - 1 : x + g0 + 1;
    o += (o < 0) ? n : 0;
    o -= (o >= n) ? n : 0;
    int base = 0;
#pragma unroll 1
    for (int g = g0; g < g1; ++g) {
        const int first = second ? o : x;
        if (g != hr || first < hn) {
            const int q = base + first;
            const float4 uo = v.u[k.sa + o];
            sa_ += cS[q];
            const float t = cH[q];
            vx = fmaf(t, uo.x, vx);
            vy = fmaf(t, uo.y, vy);
            vz = fmaf(t, uo.z, vz);
        }
        base += n;
        if (second) {
            o = (o == 0) ? n - 1 : o - 1;
        } else {
            o = (o == n - 1) ? 0 : o + 1;
        }
    }
}

// J == K, both halves of slot x's pairs in rows [g0, g1) in one walk: pair
// (x, of) with x first and pair (os, x) with x second, of advancing and os
// retreating by one per row, each half in its own sums (two independent
// chains), joined at the end
__device__ __forceinline__ void tri_visits2(const NbrView &v, const Blk &k, const float *cA, const float *cH,
                                            const float *cC, int x, int g0, int g1, float &sa_, float &vx, float &vy,
                                            float &vz)
{
    const int n = k.m, hn = n >> 1, hr = (n & 1) ? -1 : hn - 1;   // half row of an even n
    int of = x + g0 + 1, os = x - g0 - 1;
    of -= (of >= n) ? n : 0;
    os += (os < 0) ? n : 0;
    float s2 = 0.f, wx = 0.f, wy = 0.f, wz = 0.f;
    int base = 0;
#pragma unroll 1
    for (int g = g0; g < g1; ++g) {
        const bool half = (g == hr);
        if (!half || x < hn) {
            const int q = base + x;
            const float4 uo = v.u[k.sa + of];
            sa_ += cA[q];
            const float t = cH[q];
            vx = fmaf(t, uo.x, vx);
            vy = fmaf(t, uo.y, vy);
            vz = fmaf(t, uo.z, vz);
        }
        if (!half || os < hn) {
            const int q = base + os;
            const float4 uo = v.u[k.sa + os];
            s2 += cC[q];
            const float t = cH[q];
            wx = fmaf(t, uo.x, wx);
            wy = fmaf(t, uo.y, wy);
            wz = fmaf(t, uo.z, wz);
        }
        base += n;
        of = (of == n - 1) ? 0 : of + 1;
        os = (os == 0) ? n - 1 : os - 1;
    }
    sa_ += s2;
    vx += wx;
    vy += wy;
    vz += wz;
}

__device__ inline void force_slots(const NbrView &v, const Blk &k, int g0, int g1, int lane)
{
    const float *cA = v.pc, *cH = v.pc + v.pcs, *cC = v.pc + 2 * v.pcs;
    if (k.tri) {
        const int n = k.m;
        if (n <= 16) {
            // lane x sums slot x's first-member pairs, lane n + x its
            // second-member pairs; the halves meet by a shuffle
            const bool second = lane >= n;
            const int x = second ? lane - n : lane;
            float sa_ = 0.f, vx = 0.f, vy = 0.f, vz = 0.f;
            if (lane < 2 * n) tri_visits(v, k, second ? cC : cA, cH, x, second, g0, g1, sa_, vx, vy, vz);
            sa_ += __shfl_down_sync(NNP_FULL, sa_, n);
            vx += __shfl_down_sync(NNP_FULL, vx, n);
            vy += __shfl_down_sync(NNP_FULL, vy, n);
            vz += __shfl_down_sync(NNP_FULL, vz, n);
            if (lane < n) slot_add(v, k.sa + x, v.u[k.sa + x], sa_, vx, vy, vz);
            return;
        }
        for (int x = lane; x < n; x += 32) {
            float sa_ = 0.f, vx = 0.f, vy = 0.f, vz = 0.f;
            tri_visits2(v, k, cA, cH, cC, x, g0, g1, sa_, vx, vy, vz);
            slot_add(v, k.sa + x, v.u[k.sa + x], sa_, vx, vy, vz);
        }
        return;
    }
    // J != K: pair (g, f) at (g - g0) s + f couples row slot sa + g with
    // column slot sb + f.  A row owner reads its row (stride 1; row owners
    // side by side at the odd stride s), a column owner one entry per row
    // (stride s; column owners side by side).  Row and column owners run the
    // same loop: slot sl walks its j-th pair at coefficient stride qs.
    const int nr = g1 - g0, nslots = nr + k.nb;
    for (int sl = lane; sl < nslots; sl += 32) {
        const bool is_row = sl < nr;
        const int slot = is_row ? k.sa + g0 + sl : k.sb + (sl - nr);
        const float4 us = v.u[slot];
        const int cnt = is_row ? k.nb : nr;
        const int q0 = is_row ? sl * k.s : sl - nr;
        const int qs = is_row ? 1 : k.s;
        const float *c1p = is_row ? cA : cC;
        const float4 *up = v.u + (is_row ? k.sb : k.sa + g0);
        float sa_ = 0.f, vx = 0.f, vy = 0.f, vz = 0.f;
#pragma unroll 2
        for (int j = 0; j < cnt; ++j) {
            const int q = q0 + j * qs;
            const float4 uo = up[j];
            sa_ += c1p[q];
            const float bt = cH[q];
            vx = fmaf(bt, uo.x, vx);
            vy = fmaf(bt, uo.y, vy);
            vz = fmaf(bt, uo.z, vz);
        }
        slot_add(v, slot, us, sa_, vx, vy, vz);
    }
}

// Network of one type in the packed float layout of wpar: inpw[nin],
// inpb[nin], outw[nout], outb[nout], then per layer the bias[no] and the
// transposed weights W^T[m * wt_stride(no) + n] = W[n][m].
struct NetView {
    const float *inpw, *inpb, *outw, *outb;
    const float *b[NNP_MAX_LAYERS];
    const float *wt[NNP_MAX_LAYERS];
    int ws[NNP_MAX_LAYERS];   // row stride of W^T
};

__device__ inline NetView net_view(const float *base, const DevType &T)
{
    NetView v;
    const float *p = base;
    const int nin = T.nodes[0], nout = T.nodes[T.nlayer];
    v.inpw = p; p += nin;
    v.inpb = p; p += nin;
    v.outw = p; p += nout;
    v.outb = p; p += nout;
    for (int l = 0; l < T.nlayer; ++l) {
        const int ni = T.nodes[l], no = T.nodes[l + 1];
        v.b[l] = p; p += no;
        v.ws[l] = wt_stride(no);
        v.wt[l] = p; p += (i64)ni * v.ws[l];
    }
    return v;
}

// Prebuilt path: every angular block goes through the generic code above.
struct GenericBlocks {
    template <typename Acc>
    // Gb: the block's first symmetry function in the atom's row; eb: its first dE/dG
    __device__ static bool symm(const NbrView &, int, int, const Blk &, int, int, float *) { return false; }
    __device__ static bool force(const NbrView &, int, int, const Blk &, int, int, int, int, int, const float *)
    {
        return false;
    }
    __device__ static bool tangent(const NbrView &, int, int, const Blk &, int, int, float *) { return false; }
    // radial term of one neighbour in the force kernel
    __device__ static bool radial_force(int, int, float, float, float, const float *, float &) { return false; }
    // one lane's radial sum in the symmetry-function kernel (radial_sum)
    template <typename Acc>
    __device__ static bool radial_symm(int, const NbrView &, const float *, float, float, int, int, int, Acc &)
    {
        return false;
    }
    // one lane's radial tangent sum in the training tangent kernel (radial_tangent_sum)
    __device__ static bool radial_tangent(int, const NbrView &, const float *, const float *, const float *, float,
                                          float, int, int, int, float &)
    {
        return false;
    }
};

// Radial function (rs, eta) of a block whose form is known at compile time,
// summed over neighbour slots k0, k0 + G, ... < s1 (fcv: the block's cutoff
// values): the generic loop with the form switch resolved outside it.  Each
// term is rounded before it is added (no multiply-add contraction across
// the two), as in the generic loop, so both give the same sums bit for bit.
__device__ __forceinline__ void acc_term(float &acc, float v) { acc = __fadd_rn(acc, v); }
__device__ __forceinline__ void acc_term(double &acc, float v) { acc += (double)v; }
// The tangent kernel's sum of G'(r) rr over the same slots (fdv: cutoff
// slopes, rr: rates of change of the distances), form fixed at compile time.
template <int FORM>
__device__ __forceinline__ float radial_tangent_sum(const NbrView &v, const float *fcv, const float *fdv,
                                                   const float *rr, float rs, float eta, int k0, int s1, int G)
{
    float acc = 0.f;
    for (int k = k0; k < s1; k += G) {
        float val, der;
        radial_fd(FORM, v.r[k], rs, eta, fcv[k], fdv[k], val, der);
        acc = fmaf(der, rr[k], acc);
    }
    return acc;
}

template <int FORM, typename Acc>
__device__ __forceinline__ Acc radial_sum(const NbrView &v, const float *fcv, float rs, float eta, int k0, int s1,
                                          int G)
{
    Acc acc = 0;
    for (int k = k0; k < s1; k += G) {
        float val, der;
        radial_fd(FORM, v.r[k], rs, eta, fcv[k], 0.f, val, der);
        acc_term(acc, val);
    }
    return acc;
}

// ---------------------------------------------------------------- kernel bodies

// Symmetry functions of atoms [warp-strided]: NNP::compute_symm (nnp/nnp.cpp:350-392).
// Radial: lanes own functions and walk their neighbour-type segment.  Angular:
// one (J,K) block at a time, lanes over the block's pairs.  Blocks::symm may
// take over a block with code specialised for it.
// Atoms are visited in `order` (grouped by element), so at any time the SMs
// run one element's block code, which keeps the instruction working set small.
template <typename Acc, class Blocks>
__device__ void symm_body(i64 N, const DevPot *__restrict__ pot, const float2 *__restrict__ rpar,
                          const float4 *__restrict__ apar, const int *__restrict__ type, const int *__restrict__ order,
                          const float4 *__restrict__ nbr, const int *__restrict__ nbr_cnt, int cap, int ncut_max,
                          int ndamp_max, int gstride, float *__restrict__ G, float *smem)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int per = nbr_view_floats(cap, ncut_max, ndamp_max, gstride, false, NNP_FORCE_CHUNK);
    const NbrView v = nbr_view(smem + (size_t)warp * ((per + 3) & ~3), cap, ncut_max, ndamp_max, gstride, false);
    const DevPot &P = *pot;
    for (i64 idx = blockIdx.x * (i64)NNP_WARPS + warp; idx < N; idx += (i64)gridDim.x * NNP_WARPS) {
        const i64 i = order[idx];
        const int II = type[i];
        if ((unsigned)II >= (unsigned)P.ntypes) continue;        // type out of range (reported by the call)
        const DevType &T = P.t[II];
        stage_records(v, nbr + i * cap, nbr_cnt[i], cap, P, T, lane);
        float *Gi = G + i * gstride;
        for (int g = lane; g < gstride; g += 32) Gi[g] = 0.f;
        __syncwarp();
        for (int J = 0; J < P.ntypes; ++J) {
            const DevBlockR B = T.br[J];
            if (B.n == 0) continue;
            const int s0 = v.seg[J], s1 = v.seg[J + 1];
            int f, ph, G;
            radial_lanes(B.n, lane, f, ph, G);
            Acc acc = 0;
            if (f < B.n) {
                const float2 q = rpar[B.par + f];
                if (!Blocks::template radial_symm<Acc>(B.form, v, v.fc + B.cut * cap, q.x, q.y, s0 + ph, s1, G, acc))
                    for (int k = s0 + ph; k < s1; k += G) {
                        float val, der;
                        radial_fd(B.form, v.r[k], q.x, q.y, v.fc[B.cut * cap + k], v.fd[B.cut * cap + k], val, der);
                        acc_add(acc, val, 1.f);
                    }
            }
            for (int off = 1; off < G; off <<= 1) acc += __shfl_xor_sync(NNP_FULL, acc, off);
            if (ph == 0 && f < B.n) Gi[B.off_g + f] = (float)acc;
        }
        // angular blocks tt = K (K + 1) / 2 + J, J <= K
        for (int K = 0, tt = 0; K < P.ntypes; ++K)
        for (int J = 0; J <= K; ++J, ++tt) {
            const DevBlockA B = T.ba[tt];
            if (B.n == 0) continue;
            Blk k;
            if (!make_blk(v, J, K, k)) continue;
            if (!Blocks::template symm<Acc>(v, II, tt, k, cap, lane, Gi + B.off_g)) {
                for (int f = lane; f < B.n; f += 32) v.par[f] = apar[B.par + f];
                __syncwarp();
                symm_block_generic<Acc>(v, B, k, cap, lane, Gi);
            }
            __syncwarp();
        }
        __syncwarp();
    }
}

// Forces: NNP::compute_force (nnp/nnp.cpp:412-476).  With e = dE_i/dG_i, every
// pair and triplet contributes dE_i/dd_j for the neighbour displacements
// d_j = x_i - x_j - R q.  For a triplet (a,b) with dE/dcos = hc,
// dE/dr_a = hra, dE/dr_b = hrb:
//   dE/dd_a = (hra - hc cos/r_a) u_a + (hc/r_a) u_b,  and a <-> b.
// The pair pass writes three coefficients per pair into shared memory
// (hra - hc cos/r_a, hc, hrb - hc cos/r_b), then each lane owns neighbour slots
// and sums their pairs in a fixed order (no atomics), scaling the sum of the
// hc u_partner terms by its own 1/r at the end.  Finally F_j += g_j and F_i -= sum_j g_j in FP64: the
// Newton-3 scatter of nnp.cpp:443-471.
template <class Blocks>
__device__ void force_body(i64 N, const DevPot *__restrict__ pot, const float2 *__restrict__ rpar,
                           const float4 *__restrict__ apar, const int *__restrict__ type, const int *__restrict__ order,
                           const float4 *__restrict__ nbr, const int *__restrict__ nbr_cnt, int cap, int ncut_max,
                           int ndamp_max, int gstride, const float *__restrict__ dEdG, double *__restrict__ F,
                           DevErr *err, float *smem, const int *__restrict__ atom_struct = nullptr,
                           double *__restrict__ vir = nullptr)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int per = nbr_view_floats(cap, ncut_max, ndamp_max, gstride, true, NNP_FORCE_CHUNK);
    const NbrView v = nbr_view(smem + (size_t)warp * ((per + 3) & ~3), cap, ncut_max, ndamp_max, gstride, true);
    const DevPot &P = *pot;
    const i64 stride = (i64)gridDim.x * NNP_WARPS, idx0 = blockIdx.x * (i64)NNP_WARPS + warp;
    // load pipeline (pack_nt): atom idx (i0, nt0) is in shared memory, atom
    // idx + stride (i1, nt1) known, atom idx + 2 stride (i2) indexed
    auto row_len = [&](int nt) { return ((nt & 15) < P.ntypes) ? P.t[nt & 15].n_input : 0; };
    int i0 = 0, nt0 = 0, i1 = 0, nt1 = 0, i2 = 0;
    if (idx0 < N) {
        i0 = order[idx0];
        nt0 = pack_nt(nbr_cnt[i0], type[i0]);
        prefetch_rows(v.raw, nbr + (i64)i0 * cap, nt0 >> 4, v.vec, dEdG + (i64)i0 * gstride, row_len(nt0), lane);
    }
    if (idx0 + stride < N) {
        i1 = order[idx0 + stride];
        nt1 = pack_nt(nbr_cnt[i1], type[i1]);
    }
    if (idx0 + 2 * stride < N) i2 = order[idx0 + 2 * stride];
    for (i64 idx = idx0; idx < N; idx += stride) {
        const i64 i = i0;
        const int II = nt0 & 15;
        // loads for two and three atoms on, used by later iterations
        const int nt2 = (idx + 2 * stride < N) ? pack_nt(nbr_cnt[i2], type[i2]) : 0;
        const int i3 = (idx + 3 * stride < N) ? order[idx + 3 * stride] : 0;
        const float *vc = v.vec;
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncwarp();
        const bool ok = II < P.ntypes;                          // else type out of range (reported by the call)
        const int n = ok ? stage_records(v, v.raw, nt0 >> 4, cap, P, P.t[II], lane) : 0;
        // the next atom's records and dE/dG row stream in meanwhile
        const bool more = idx + stride < N;
        const int in = i1, ntn = nt1;
        if (more) prefetch_rows(v.raw, nbr + (i64)i1 * cap, nt1 >> 4, nullptr, nullptr, 0, lane);
        i0 = i1;
        nt0 = nt1;
        i1 = i2;
        nt1 = nt2;
        i2 = i3;
        if (!ok) {
            if (more) prefetch_rows(nullptr, nullptr, 0, v.vec, dEdG + (i64)in * gstride, row_len(ntn), lane);
            continue;
        }
        const DevType &T = P.t[II];
        // radial: lanes own their neighbour slot (initialises g)
        for (int k = lane; k < n; k += 32) {
            const int tk = v.t[k];
            const DevBlockR B = T.br[tk];
            const float4 u = v.u[k];
            const float fc = v.fc[B.cut * cap + k], fd = v.fd[B.cut * cap + k];
            float amp = 0.f;
            if (!Blocks::radial_force(II, tk, v.r[k], fc, fd, vc + B.off_g, amp)) {
                for (int f = 0; f < B.n; ++f) {
                    const float2 q = rpar[B.par + f];
                    float val, der;
                    radial_fd(B.form, v.r[k], q.x, q.y, fc, fd, val, der);
                    amp = fmaf(vc[B.off_g + f], der, amp);
                }
            }
            v.gx[k] = amp * u.x;
            v.gy[k] = amp * u.y;
            v.gz[k] = amp * u.z;
        }
        __syncwarp();
        // angular blocks tt = K (K + 1) / 2 + J, J <= K
        for (int K = 0, tt = 0; K < P.ntypes; ++K)
        for (int J = 0; J <= K; ++J, ++tt) {
            const DevBlockA B = T.ba[tt];
            if (B.n == 0) continue;
            Blk k;
            if (!make_blk(v, J, K, k)) continue;
            bool staged = false;
            const int R = chunk_rows(k);
            for (int g0 = 0; g0 < k.rows; g0 += R) {
                const int g1 = min(k.rows, g0 + R);
                const int c0 = g0 * k.m, c1 = min(k.npairs, g1 * k.m), qoff = g0 * k.s;
                if (!Blocks::force(v, II, tt, k, c0, c1, qoff, cap, lane, vc + B.off_g)) {
                    if (!staged) {
                        for (int f = lane; f < B.n; f += 32) v.par[f] = apar[B.par + f];
                        __syncwarp();
                        staged = true;
                    }
                    force_pairs_generic(v, B, vc + B.off_g, k, c0, c1, qoff, cap, lane);
                }
                __syncwarp();
                force_slots(v, k, g0, g1, lane);
                __syncwarp();
            }
        }
        __syncwarp();
        // the next atom's dE/dG row streams in during the scatter
        if (more) prefetch_rows(nullptr, nullptr, 0, v.vec, dEdG + (i64)in * gstride, row_len(ntn), lane);
        // scatter: F_j += g_j, F_i -= sum g_j
        double fx = 0.0, fy = 0.0, fz = 0.0;
        bool bad = false;
        for (int k = lane; k < n; k += 32) {
            const double gx = v.gx[k], gy = v.gy[k], gz = v.gz[k];
            bad |= !(finite_d(gx) && finite_d(gy) && finite_d(gz));
            const i64 j = v.j[k];
            atomicAdd(&F[3 * j], gx);
            atomicAdd(&F[3 * j + 1], gy);
            atomicAdd(&F[3 * j + 2], gz);
            fx += gx;
            fy += gy;
            fz += gz;
        }
        fx = warp_sum(fx);
        fy = warp_sum(fy);
        fz = warp_sum(fz);
        if (lane == 0) {
            atomicAdd(&F[3 * i], -fx);
            atomicAdd(&F[3 * i + 1], -fy);
            atomicAdd(&F[3 * i + 2], -fz);
        }
        if (vir) {
            // virial W = -dE/d(strain): under x -> (I + e) x every displacement
            // d_k = x_i - x_j - R q becomes (I + e) d_k, so W_ab = -sum_k g_a d_b
            double w[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int k = lane; k < n; k += 32) {
                const double g3[3] = {v.gx[k], v.gy[k], v.gz[k]};
                const float4 u = v.u[k];
                const double r = v.r[k];
                const double d3[3] = {u.x * r, u.y * r, u.z * r};
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int b = 0; b < 3; ++b) w[3 * a + b] -= g3[a] * d3[b];
            }
#pragma unroll
            for (int q = 0; q < 9; ++q) w[q] = warp_sum(w[q]);
            if (lane == 0) {
                double *ws = vir + 9 * (i64)atom_struct[i];
#pragma unroll
                for (int q = 0; q < 9; ++q) atomicAdd(ws + q, w[q]);
            }
        }
        if (__any_sync(NNP_FULL, bad) && lane == 0) atomicMax(&err->nonfinite, 1);
        __syncwarp();
    }
}

// Tangent of the symmetry functions along a displacement field V (training
// force term): C_i = sum_k dG_i/dx_k . V_k from the staged neighbour geometry,
// the force kernel's basis derivatives contracted with the relative
// displacements V_i - V_k instead of scattered.  Blocks::tangent may take
// over a block with code specialised for it.
template <class Blocks>
__device__ void tangent_body(i64 N, const DevPot *__restrict__ pot, const float2 *__restrict__ rpar,
                             const float4 *__restrict__ apar, const int *__restrict__ type, const int *__restrict__ order,
                             const float4 *__restrict__ nbr, const int *__restrict__ nbr_cnt, int cap, int ncut_max,
                             int ndamp_max, int gstride, const float4 *__restrict__ V, float *__restrict__ Cout,
                             float *smem)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int per = nbr_view_floats(cap, ncut_max, ndamp_max, gstride, true, NNP_FORCE_CHUNK);
    const NbrView v = nbr_view(smem + (size_t)warp * ((per + 3) & ~3), cap, ncut_max, ndamp_max, gstride, true);
    // the force view's per-neighbour gradient arrays hold the relative
    // displacement dv_k = V_i - V_k, and its pair-coefficient area the rate
    // of change of the distance, rr_k = u_k . dv_k (cap <= 3 pcs)
    float *rr = v.pc;
    const DevPot &P = *pot;
    const i64 stride = (i64)gridDim.x * NNP_WARPS, idx0 = blockIdx.x * (i64)NNP_WARPS + warp;
    i64 i_next = 0;
    int n_next = 0;
    prefetch_atom(v, idx0, N, order, nbr, nbr_cnt, cap, lane, i_next, n_next);
    for (i64 idx = idx0; idx < N; idx += stride) {
        const i64 i = i_next;
        const int II = type[i];
        if ((unsigned)II >= (unsigned)P.ntypes) {               // type out of range (reported by the call)
            asm volatile("cp.async.wait_group 0;" ::: "memory");
            __syncwarp();
            prefetch_atom(v, idx + stride, N, order, nbr, nbr_cnt, cap, lane, i_next, n_next);
            continue;
        }
        const DevType &T = P.t[II];
        const int n = stage_prefetched(v, n_next, cap, P, T, lane);
        prefetch_atom(v, idx + stride, N, order, nbr, nbr_cnt, cap, lane, i_next, n_next);
        const float4 vi = V[i];
        for (int k = lane; k < n; k += 32) {
            const float4 vk = V[v.j[k]];
            const float dx = vi.x - vk.x, dy = vi.y - vk.y, dz = vi.z - vk.z;
            v.gx[k] = dx;
            v.gy[k] = dy;
            v.gz[k] = dz;
            const float4 u = v.u[k];
            rr[k] = u.x * dx + u.y * dy + u.z * dz;
        }
        float *Ci = Cout + i * gstride;
        for (int g = lane; g < gstride; g += 32) Ci[g] = 0.f;
        __syncwarp();
        // radial: dG/deps = G'(r) rr
        for (int J = 0; J < P.ntypes; ++J) {
            const DevBlockR B = T.br[J];
            if (B.n == 0) continue;
            const int s0 = v.seg[J], s1 = v.seg[J + 1];
            int f, ph, G;
            radial_lanes(B.n, lane, f, ph, G);
            float acc = 0.f;
            if (f < B.n) {
                const float2 q = rpar[B.par + f];
                if (!Blocks::radial_tangent(B.form, v, v.fc + B.cut * cap, v.fd + B.cut * cap, rr, q.x, q.y, s0 + ph, s1,
                                            G, acc))
                    for (int k = s0 + ph; k < s1; k += G) {
                        float val, der;
                        radial_fd(B.form, v.r[k], q.x, q.y, v.fc[B.cut * cap + k], v.fd[B.cut * cap + k], val, der);
                        acc = fmaf(der, rr[k], acc);
                    }
            }
            for (int off = 1; off < G; off <<= 1) acc += __shfl_xor_sync(NNP_FULL, acc, off);
            if (ph == 0 && f < B.n) Ci[B.off_g + f] = acc;
        }
        __syncwarp();
        // angular: dG/deps = dG/dcos dcos + dG/dr_a rr_a + dG/dr_b rr_b with
        // dcos = (u_b . dv_a - cos rr_a)/r_a + (u_a . dv_b - cos rr_b)/r_b
        // angular blocks tt = K (K + 1) / 2 + J, J <= K
        for (int K = 0, tt = 0; K < P.ntypes; ++K)
        for (int J = 0; J <= K; ++J, ++tt) {
            const DevBlockA B = T.ba[tt];
            if (B.n == 0) continue;
            Blk k;
            if (!make_blk(v, J, K, k)) continue;
            if (Blocks::tangent(v, II, tt, k, cap, lane, Ci + B.off_g)) {
                __syncwarp();
                continue;
            }
            for (int f = lane; f < B.n; f += 32) v.par[f] = apar[B.par + f];
            __syncwarp();
            for (int f0 = 0; f0 < B.n; f0 += NNP_SYMM_CHUNK) {
                const int nf = min(NNP_SYMM_CHUNK, B.n - f0);
                float acc[NNP_SYMM_CHUNK];
#pragma unroll
                for (int f = 0; f < NNP_SYMM_CHUNK; ++f) acc[f] = 0.f;
                PairIt it = pit_init(k, lane);
#pragma unroll 1
                for (int p = lane; p < k.npairs; p += 32, pit_next(k, it)) {
                    int a, b;
                    pit_slots(k, it, a, b);
                    const float4 ua = v.u[a], ub = v.u[b];
                    const float cs = ua.x * ub.x + ua.y * ub.y + ua.z * ub.z;
                    const float uba = ub.x * v.gx[a] + ub.y * v.gy[a] + ub.z * v.gz[a];
                    const float uab = ua.x * v.gx[b] + ua.y * v.gy[b] + ua.z * v.gz[b];
                    const float ra = rr[a], rb = rr[b];
                    const float dcos = (uba - cs * ra) * ua.w + (uab - cs * rb) * ub.w;
                    const float fca = v.fc[B.cut * cap + a], fcb = v.fc[B.cut * cap + b];
                    const float fda = v.fd[B.cut * cap + a], fdb = v.fd[B.cut * cap + b];
#pragma unroll
                    for (int f = 0; f < NNP_SYMM_CHUNK; ++f) {
                        if (f < nf) {
                            const float4 q = v.par[f0 + f];
                            const int iz = (__float_as_int(q.w) >> 8) - 1;
                            float h, hc, hra, hrb;
                            angular_generic(B.form, v.r[a], v.r[b], cs, fca, fcb, fda, fdb, q.x, q.y, iz, q.z, true, h,
                                            hc, hra, hrb);
                            acc[f] = fmaf(hc, dcos, fmaf(hra, ra, fmaf(hrb, rb, acc[f])));
                        }
                    }
                }
#pragma unroll
                for (int f = 0; f < NNP_SYMM_CHUNK; ++f) {
                    if (f < nf) {
                        const float s = warp_sum(acc[f]);
                        if (lane == 0) Ci[B.off_g + f0 + f] = s;
                    }
                }
            }
            __syncwarp();
        }
        __syncwarp();
    }
}

#endif  // __CUDACC__

}  // namespace nnp
