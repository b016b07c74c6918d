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
