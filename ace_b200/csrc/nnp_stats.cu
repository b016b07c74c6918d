// nnp_stats.cu -- input statistics of the atomic networks over a training set.
//
// NNPTEFR::train's input statistics (nnptefr.cpp:689-781) on the device: for
// every element and every network input (symmetry function) the count of
// atoms, the largest and smallest value, the harmonic mean N / sum(1/G),
// the mean, the standard deviation sqrt(sum (mean - G)^2 / (N - 1)) and the
// root mean square sqrt(sum G^2 / N), over all atoms of the batch.  They set
// the networks' input bias and scale (PREBIAS / PRESCALE, nnptefr.cpp:783-880).
//
// The atoms of an element are a contiguous range of `order` after the
// neighbour stage, so each statistic is a segmented reduction: a block owns
// 32 inputs (one per lane) of one element and one of STAT_PARTS equal parts
// of its atoms, warps stride over the atoms and meet in shared memory in a
// fixed order.  The parts are summed on the host in a fixed order too, so
// the results do not depend on scheduling.  Sums are FP64; the symmetry
// functions are the FP32 rows the energy path computes.
#include <cfloat>

#include "../../include/nnp_b200.h"
#include "nnp_device.cuh"
#include "nnp_engine.h"

namespace nnp {

namespace {

constexpr int STAT_PARTS = 64;     // parts of each element's atoms (blocks per 32 inputs)
constexpr int STAT_WARPS = 8;
constexpr int NSTAT1 = 5;          // first pass: max, min, sum 1/G, sum G, sum G^2
constexpr int NSTAT = 6;           // per (element, input) in the partial buffer: the first pass + sum (mean - G)^2

// pass 0: max, min, sum 1/G, sum G, sum G^2; pass 1: sum (mean - G)^2
__global__ void __launch_bounds__(STAT_WARPS * 32) k_input_stats(int pass, const float *__restrict__ G, int gstride,
                                                                 const int *__restrict__ order,
                                                                 const int *__restrict__ type_count,
                                                                 const DevPot *__restrict__ pot,
                                                                 const double *__restrict__ mean,
                                                                 double *__restrict__ part)
{
    __shared__ double red[STAT_WARPS][32][NSTAT1];
    const int T = blockIdx.z, p = blockIdx.y, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int k = blockIdx.x * 32 + lane;
    const int nin = pot->t[T].n_input;
    int base = 0;
    for (int t = 0; t < T; ++t) base += type_count[t];
    const int cnt = type_count[T];
    const int lo = base + (int)((int64_t)cnt * p / STAT_PARTS), hi = base + (int)((int64_t)cnt * (p + 1) / STAT_PARTS);
    double a0 = pass == 0 ? -DBL_MAX : 0.0, a1 = pass == 0 ? DBL_MAX : 0.0, a2 = 0.0, a3 = 0.0, a4 = 0.0;
    if (k < nin) {
        const double m = pass == 1 ? mean[(size_t)T * gstride + k] : 0.0;
        for (int idx = lo + warp; idx < hi; idx += STAT_WARPS) {
            const double g = G[(int64_t)order[idx] * gstride + k];
            if (pass == 0) {
                a0 = fmax(a0, g);
                a1 = fmin(a1, g);
                a2 += 1.0 / g;
                a3 += g;
                a4 += g * g;
            } else {
                const double d = m - g;
                a0 += d * d;
            }
        }
    }
    red[warp][lane][0] = a0;
    red[warp][lane][1] = a1;
    red[warp][lane][2] = a2;
    red[warp][lane][3] = a3;
    red[warp][lane][4] = a4;
    __syncthreads();
    if (warp == 0 && k < nin) {
        double r0 = red[0][lane][0], r1 = red[0][lane][1], r2 = red[0][lane][2], r3 = red[0][lane][3],
               r4 = red[0][lane][4];
        for (int w = 1; w < STAT_WARPS; ++w) {
            if (pass == 0) {
                r0 = fmax(r0, red[w][lane][0]);
                r1 = fmin(r1, red[w][lane][1]);
                r2 += red[w][lane][2];
                r3 += red[w][lane][3];
                r4 += red[w][lane][4];
            } else {
                r0 += red[w][lane][0];
            }
        }
        double *o = part + (((size_t)T * STAT_PARTS + p) * gstride + k) * NSTAT;
        if (pass == 0) {
            o[0] = r0;
            o[1] = r1;
            o[2] = r2;
            o[3] = r3;
            o[4] = r4;
        } else {
            o[5] = r0;
        }
    }
}

}  // namespace

// Statistics of the symmetry functions in E.G over the centres of the last
// step (E.order / E.type_fill must be those of that step).  count[T] atoms
// per element; stats[(T * NNP_NSTATS + s) * gstride + k] for statistic s
// (NNP_STAT_*) of input k.  Returns "" or an error.
std::string run_input_stats(Engine &E, std::vector<int64_t> &count, std::vector<double> &stats)
{
    const int T = E.dpot.ntypes, gs = E.gstride;
    DBuf<double> part, mean;
    cudaError_t e = part.reserve((size_t)T * STAT_PARTS * gs * NSTAT);
    if (e == cudaSuccess) e = mean.reserve((size_t)T * gs);
    if (e != cudaSuccess) {
        part.release();
        mean.release();
        return std::string("device allocation failed: ") + cudaGetErrorString(e);
    }
    std::vector<int> tc(T + 1, 0);
    e = cudaMemcpyAsync(tc.data(), E.type_fill.p, sizeof(int) * T, cudaMemcpyDeviceToHost, E.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(part.p, 0, sizeof(double) * (size_t)T * STAT_PARTS * gs * NSTAT, E.stream);
    const dim3 grid((gs + 31) / 32, STAT_PARTS, T);
    if (e == cudaSuccess && T > 0) {
        k_input_stats<<<grid, STAT_WARPS * 32, 0, E.stream>>>(0, E.G.p, gs, E.order.p, E.type_fill.p, E.d_pot, nullptr,
                                                            part.p);
        E.launches += 1;
        e = cudaGetLastError();
    }
    std::vector<double> hp((size_t)T * STAT_PARTS * gs * NSTAT);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(hp.data(), part.p, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, E.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E.stream);
    if (e != cudaSuccess) {
        part.release();
        mean.release();
        return std::string("input statistics: ") + cudaGetErrorString(e);
    }
    count.assign(T, 0);
    stats.assign((size_t)T * NNP_NSTATS * gs, 0.0);
    std::vector<double> mh((size_t)T * gs, 0.0);
    auto S = [&](int t, int s, int k) -> double & { return stats[((size_t)t * NNP_NSTATS + s) * gs + k]; };
    for (int t = 0; t < T; ++t) {
        count[t] = tc[t];
        const int nin = E.dpot.t[t].n_input;
        for (int k = 0; k < nin; ++k) {
            double mx = -DBL_MAX, mn = DBL_MAX, hs = 0, s1 = 0, s2 = 0;
            for (int p = 0; p < STAT_PARTS; ++p) {
                const double *o = &hp[(((size_t)t * STAT_PARTS + p) * gs + k) * NSTAT];
                mx = std::max(mx, o[0]);
                mn = std::min(mn, o[1]);
                hs += o[2];
                s1 += o[3];
                s2 += o[4];
            }
            const double n = (double)tc[t];
            S(t, NNP_STAT_MAX, k) = mx;
            S(t, NNP_STAT_MIN, k) = mn;
            S(t, NNP_STAT_HARMONIC, k) = n / hs;
            S(t, NNP_STAT_MEAN, k) = s1 / n;
            S(t, NNP_STAT_RMS, k) = std::sqrt(s2 / n);
            mh[(size_t)t * gs + k] = s1 / n;
        }
    }
    // second pass: deviations from the mean (two passes, as the reference)
    e = cudaMemcpyAsync(mean.p, mh.data(), sizeof(double) * mh.size(), cudaMemcpyHostToDevice, E.stream);
    if (e == cudaSuccess && T > 0) {
        k_input_stats<<<grid, STAT_WARPS * 32, 0, E.stream>>>(1, E.G.p, gs, E.order.p, E.type_fill.p, E.d_pot, mean.p,
                                                            part.p);
        E.launches += 1;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(hp.data(), part.p, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, E.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E.stream);
    part.release();
    mean.release();
    if (e != cudaSuccess) return std::string("input statistics: ") + cudaGetErrorString(e);
    for (int t = 0; t < T; ++t)
        for (int k = 0; k < E.dpot.t[t].n_input; ++k) {
            double v = 0;
            for (int p = 0; p < STAT_PARTS; ++p) v += hp[(((size_t)t * STAT_PARTS + p) * gs + k) * NSTAT + 5];
            S(t, NNP_STAT_DEV, k) = std::sqrt(v / ((double)tc[t] - 1.0));
        }
    return "";
}

}  // namespace nnp

// ------------------------------------------------------------------ Taylor expansion of the training set
//
// NNPTEFR's force perturbation (nnptefr.cpp:2733-2830): every structure whose
// mean force norm exceeds 1e-12 gets nadd copies in which each atom moves by
// dr = vr (sin t cos p, sin t sin p, cos t), cos t and p / pi uniform in
// (-1, 1), vr drawn from a distribution of width rdelta, and the copy's
// energy is the first-order estimate E - sum_j dr_j . F_j.  The random numbers
// come from a counter-based hash of (seed, output structure, atom, draw), so
// a copy does not depend on the order in which the GPU makes it.

namespace nnp {

namespace {

__host__ __device__ inline uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// uniform double in (0, 1) of draw k of atom j of output structure o
__host__ __device__ inline double taylor_uniform(uint64_t seed, int64_t o, int64_t j, int k)
{
    const uint64_t h = mix64(mix64(mix64(seed + 0x9e3779b97f4a7c15ull) ^ (uint64_t)o) ^ ((uint64_t)j * 4 + (uint64_t)k));
    return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

// radius of the displacement: the inverse-CDF draws of rng::dist (math/random.cpp:64-146)
// with location 0 and width w
__device__ inline double taylor_radius(int dist, double w, double u1, double u2)
{
    const double pi = 3.141592653589793;
    switch (dist) {
    case 1: return u1 * w;                                                    // UNIFORM(0, w)
    case 2: { const double p = u1 - 0.5; return -w * ((p > 0) - (p < 0)) * log(1.0 - 2.0 * fabs(p)); }   // LAPLACE
    case 3: return w * sqrt(-2.0 * log(u1)) * cos(2.0 * pi * u2);            // NORMAL (Box-Muller)
    case 5: return w * 2.0 / pi * log(tan(0.5 * pi * u1));                    // SECH
    case 6: return w * log(u1 / (1.0 - u1));                                  // LOGISTIC
    case 7: {                                                                 // COSINE (the reference's fit of its inverse CDF)
        if (u1 < 0.5) {
            const double t = sqrt(-2.0 * log(u1));
            return w * (0.820251 - 0.806770 * t + 0.093247 * t * t);
        }
        const double t = sqrt(-2.0 * log(1.0 - u1));
        return -w * (0.820251 - 0.806770 * t + 0.093247 * t * t);
    }
    default: return 0.0;
    }
}

// one block per output structure: copy m of source structure src[o]
__global__ void k_taylor(const int64_t *__restrict__ off, const double *__restrict__ pos,
                         const double *__restrict__ energy, const double *__restrict__ forces,
                         const int *__restrict__ src, const int *__restrict__ copy, const int64_t *__restrict__ out_off,
                         int dist, double rdelta, uint64_t seed, double *__restrict__ out_pos,
                         double *__restrict__ out_energy)
{
    __shared__ double red[256];
    const int64_t o = blockIdx.x;
    const int s = src[o];
    const bool perturb = copy[o] > 0;
    const int64_t a0 = off[s], n = off[s + 1] - a0, b0 = out_off[o];
    double de = 0.0;
    for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
        const double *x = pos + 3 * (a0 + j);
        double *y = out_pos + 3 * (b0 + j);
        if (!perturb) {
            y[0] = x[0];
            y[1] = x[1];
            y[2] = x[2];
            continue;
        }
        const double vr = taylor_radius(dist, rdelta, taylor_uniform(seed, o, j, 0), taylor_uniform(seed, o, j, 3));
        const double ct = 2.0 * taylor_uniform(seed, o, j, 1) - 1.0, st = sqrt(1.0 - ct * ct);
        const double ph = (2.0 * taylor_uniform(seed, o, j, 2) - 1.0) * 3.141592653589793;
        const double d[3] = {vr * st * cos(ph), vr * st * sin(ph), vr * ct};
        const double *f = forces + 3 * (a0 + j);
        for (int k = 0; k < 3; ++k) y[k] = x[k] + d[k];
        de += d[0] * f[0] + d[1] * f[1] + d[2] * f[2];
    }
    red[threadIdx.x] = de;
    __syncthreads();
    for (int k = blockDim.x / 2; k; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) out_energy[o] = energy[s] - red[0];
}

}  // namespace

// Host part: the output layout (originals in order, each followed by its
// copies), the copy of the inputs to the device, the kernel and the copy
// back.  Returns "" or an error message.
std::string taylor_expand(int S, const int64_t *atom_off, const double *pos, const double *energy,
                          const double *forces, int nadd, int dist, double rdelta, uint64_t seed,
                          std::vector<int64_t> &out_off, std::vector<int> &out_src, std::vector<double> &out_pos,
                          std::vector<double> &out_energy)
{
    const int64_t N = atom_off[S];
    std::vector<int> src, cp;
    out_off.assign(1, 0);
    for (int s = 0; s < S; ++s) {
        const int64_t a0 = atom_off[s], n = atom_off[s + 1] - a0;
        double favg = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            const double *f = forces + 3 * (a0 + j);
            favg += std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
        }
        favg = n > 0 ? favg / (double)n : 0.0;
        const int copies = favg > 1.0e-12 ? nadd : 0;
        for (int m = 0; m <= copies; ++m) {
            src.push_back(s);
            cp.push_back(m);
            out_off.push_back(out_off.back() + n);
        }
    }
    const int O = (int)src.size();
    const int64_t NO = out_off.back();
    out_src = src;
    out_pos.assign(3 * (size_t)NO, 0.0);
    out_energy.assign(O, 0.0);
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return "cudaStreamCreate failed";
    DBuf<int64_t> d_off, d_oo;
    DBuf<double> d_pos, d_e, d_f, d_opos, d_oe;
    DBuf<int> d_src, d_cp;
    cudaError_t e = cudaSuccess;
    auto r = [&](cudaError_t x) { if (x != cudaSuccess && e == cudaSuccess) e = x; };
    r(d_off.reserve(S + 1));
    r(d_oo.reserve(O + 1));
    r(d_pos.reserve(3 * (size_t)std::max<int64_t>(N, 1)));
    r(d_f.reserve(3 * (size_t)std::max<int64_t>(N, 1)));
    r(d_e.reserve(S));
    r(d_opos.reserve(3 * (size_t)std::max<int64_t>(NO, 1)));
    r(d_oe.reserve(O));
    r(d_src.reserve(O));
    r(d_cp.reserve(O));
    if (e == cudaSuccess) {
        r(cudaMemcpyAsync(d_off.p, atom_off, sizeof(int64_t) * (S + 1), cudaMemcpyHostToDevice, st));
        r(cudaMemcpyAsync(d_oo.p, out_off.data(), sizeof(int64_t) * (O + 1), cudaMemcpyHostToDevice, st));
        r(cudaMemcpyAsync(d_pos.p, pos, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, st));
        r(cudaMemcpyAsync(d_f.p, forces, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, st));
        r(cudaMemcpyAsync(d_e.p, energy, sizeof(double) * S, cudaMemcpyHostToDevice, st));
        r(cudaMemcpyAsync(d_src.p, src.data(), sizeof(int) * O, cudaMemcpyHostToDevice, st));
        r(cudaMemcpyAsync(d_cp.p, cp.data(), sizeof(int) * O, cudaMemcpyHostToDevice, st));
    }
    if (e == cudaSuccess && O > 0) {
        k_taylor<<<O, 256, 0, st>>>(d_off.p, d_pos.p, d_e.p, d_f.p, d_src.p, d_cp.p, d_oo.p, dist, rdelta, seed,
                                    d_opos.p, d_oe.p);
        r(cudaGetLastError());
    }
    if (e == cudaSuccess) {
        r(cudaMemcpyAsync(out_pos.data(), d_opos.p, sizeof(double) * 3 * NO, cudaMemcpyDeviceToHost, st));
        r(cudaMemcpyAsync(out_energy.data(), d_oe.p, sizeof(double) * O, cudaMemcpyDeviceToHost, st));
        r(cudaStreamSynchronize(st));
    }
    d_off.release(); d_oo.release(); d_pos.release(); d_f.release(); d_e.release();
    d_opos.release(); d_oe.release(); d_src.release(); d_cp.release();
    cudaStreamDestroy(st);
    return e == cudaSuccess ? "" : std::string("Taylor expansion: ") + cudaGetErrorString(e);
}

}  // namespace nnp
