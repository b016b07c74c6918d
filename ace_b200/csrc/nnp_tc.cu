// nnp_tc.cu -- atomic networks on the tensor cores (tcgen05, sm_100a).
//
// Replaces k_nn_fp32 for NNP_PREC_BF16 / NNP_PREC_BF16X3: ANN::fpbp plus
// DODZ::grad (ml/nn.cpp:1402-1420, 1836-1859) for tiles of 128 atoms of one
// element.  Each hidden layer is one M=128 MMA chain per tile,
//     Z_h = A_h W_h^T          (A_0 = inpw * (G + inpb)),
// with the bias and activation applied by the thread that owns the row while
// it reads the FP32 accumulator out of TMEM.  The output layer (one neuron,
// linear) is a dot product on the CUDA cores.  The input gradient runs the
// same chain backwards,
//     D_{h-1} = (D_h W_h) * f'(z_{h-1}),   dE/dG = (D_0 W_0) * inpw,
// so a tile costs 2 (L-1) MMA chains.  Operands are BF16 in shared memory; with
// BF16X3 every operand is split into hi + lo BF16 parts and each product is
// hi*hi + hi*lo + lo*hi (FP32 accumulation), which keeps ~16 significant bits.
//
// One CTA = 4 warps; thread r owns row r of the tile (TMEM lane r).  Tiles are
// enumerated element by element over the element-sorted atom order, and a CTA
// restages its weights only when the element changes.
#include <cuda_bf16.h>

#include "nnp_device.cuh"
#include "nnp_engine.h"
#include "nnp_tc.cuh"

namespace nnp {

namespace {

constexpr int TILE = 128;
constexpr uint32_t TMEM_COLS = 128;          // widest padded layer (NNP_MAX_NODES)
constexpr uint32_t WAIT_POLLS = 1u << 26;     // default bound of one MMA-chain wait (~0.1-1 s); the final drain always uses it
constexpr int HEADER = 128;                   // mbarrier (8 B) and TMEM address slot (4 B); operands follow

__host__ __device__ inline int pad16(int n) { return (n + 15) & ~15; }

// Shared-memory plan of one network shape (identical on host and device).
struct TcPlan {
    int L;                       // layers (hidden layers = L - 1)
    int P[NNP_MAX_LAYERS + 1];   // padded widths of every layer's input
    int wf[NNP_MAX_LAYERS];      // bf16 offset of W_h   [P_{h+1} x P_h]  (forward B operand)
    int wb[NNP_MAX_LAYERS];      // bf16 offset of W_h^T [P_h x P_{h+1}]  (backward B operand)
    int wbytes;                  // bytes of one copy (hi or lo) of all weight operands
    int tile[NNP_MAX_LAYERS];    // bf16 offset of region h: A_h [128 x P_h] forward, D_h [128 x P_{h+1}] backward
    int tbytes;                  // bytes of one copy of all activation regions
    int dfloats;                 // f'(z_h) of every hidden layer, [n][128] FP32
    int vfloats;                 // inpw, inpb, hidden biases, output-layer weights (FP32, after d)
    int total;                   // bytes of the whole plan incl. the header
};

__host__ __device__ inline void make_plan(const DevType &T, bool split, TcPlan &p)
{
    p.L = T.nlayer;
    for (int l = 0; l < T.nlayer; ++l) p.P[l] = pad16(T.nodes[l]);
    int w = 0, t = 0, d = 0;
    for (int h = 0; h + 1 < p.L; ++h) {
        p.wf[h] = w;
        w += p.P[h + 1] * p.P[h];
        p.wb[h] = w;
        w += p.P[h] * p.P[h + 1];
        p.tile[h] = t;
        t += TILE * (p.P[h] > p.P[h + 1] ? p.P[h] : p.P[h + 1]);
        d += TILE * T.nodes[h + 1];
    }
    p.wbytes = w * 2;
    p.tbytes = t * 2;
    p.dfloats = d;
    int v = 2 * T.nodes[0] + T.nodes[p.L - 1];
    for (int h = 0; h + 1 < p.L; ++h) v += T.nodes[h + 1];
    p.vfloats = v;
    const int copies = split ? 2 : 1;
    p.total = HEADER + copies * (p.wbytes + p.tbytes) + 4 * (d + v);
}

struct Smem {
    __nv_bfloat16 *w_hi, *w_lo, *t_hi, *t_lo;
    float *d;
    float *vec;        // [inpw | inpb | bias of hidden layer 0, 1, ... | W_out[0][n]]
    uint64_t *bar;
    uint32_t *slot;
};

__device__ inline Smem carve(unsigned char *base, const TcPlan &p, bool split)
{
    Smem s;
    s.bar = reinterpret_cast<uint64_t *>(base);
    s.slot = reinterpret_cast<uint32_t *>(base + 8);
    unsigned char *q = base + HEADER;
    s.w_hi = reinterpret_cast<__nv_bfloat16 *>(q); q += p.wbytes;
    s.w_lo = split ? reinterpret_cast<__nv_bfloat16 *>(q) : nullptr; q += split ? p.wbytes : 0;
    s.t_hi = reinterpret_cast<__nv_bfloat16 *>(q); q += p.tbytes;
    s.t_lo = split ? reinterpret_cast<__nv_bfloat16 *>(q) : nullptr; q += split ? p.tbytes : 0;
    s.d = reinterpret_cast<float *>(q);
    s.vec = s.d + p.dfloats;
    return s;
}

// 8 consecutive values -> one 16-byte store of BF16 (hi, and the lo remainder when split)
__device__ __forceinline__ void store8(__nv_bfloat16 *hi, __nv_bfloat16 *lo, int off, const float *v)
{
    __align__(16) __nv_bfloat16 h[8], l[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        h[i] = __float2bfloat16_rn(v[i]);
        l[i] = __float2bfloat16_rn(v[i] - __bfloat162float(h[i]));
    }
    *reinterpret_cast<uint4 *>(hi + off) = *reinterpret_cast<const uint4 *>(h);
    if (lo) *reinterpret_cast<uint4 *>(lo + off) = *reinterpret_cast<const uint4 *>(l);
}

// Bias and transposed weights of layer l of a network in the wpar layout
// (net_view's layout), found by walking the layers: no per-thread pointer
// arrays, which the compiler would keep in local memory for a run-time l.
__device__ __forceinline__ void layer_ptrs(const float *net, const DevType &T, int l, const float *&b, const float *&wt,
                                           int &ws)
{
    const float *q = net + 2 * T.nodes[0] + 2 * T.nodes[T.nlayer];
    for (int m = 0; m < l; ++m) q += T.nodes[m + 1] + (i64)T.nodes[m] * wt_stride(T.nodes[m + 1]);
    b = q;
    wt = q + T.nodes[l + 1];
    ws = wt_stride(T.nodes[l + 1]);
}

// Activation and slope in the epilogues: tanh inline, the other forms through
// one out-of-line copy of the generic switch, so the unrolled epilogue loops
// stay small (instruction fetch limited the kernel).
__device__ __noinline__ void activation_call(int neuron, float c, float z, float &a, float &d)
{
    float d2;
    activation(neuron, c, z, a, d, d2);
}

__device__ __forceinline__ void tc_activation(int neuron, float c, float z, float &a, float &d)
{
    if (neuron == NEU_TANH) {
        const float t = tanhf(c * z);
        a = t;
        d = c * (1.f - t * t);
    } else {
        activation_call(neuron, c, z, a, d);
    }
}

// One MMA chain D[128 x N] = A[128 x K] * B[N x K]^T issued by thread 0 and
// waited for by every thread, at most `polls` tests of the barrier each.
// The result is the same in every thread of the block (a wait that gave up
// in any thread fails it for all), so the block leaves its tile loop as one
// and no thread is left at a barrier the others skip.  On failure the phase
// is not advanced: the drain before the TMEM release waits for that chain.
__device__ bool gemm(const Smem &s, int a_off, int b_off, int K, int N, bool split, uint32_t tmem, uint32_t &phase,
                     uint32_t polls)
{
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0) {
        tc::fence_after_sync();
        const uint32_t id = tc::idesc_bf16(TILE, N);
        const uint32_t sbo = (K / 8) * 128;
        const uint32_t a_hi = tc::smem_u32(s.t_hi + a_off), b_hi = tc::smem_u32(s.w_hi + b_off);
        uint32_t acc = 0;
        for (int kk = 0; kk < K / 16; ++kk) {
            const uint64_t ad = tc::sdesc(a_hi + kk * 256, 128, sbo);
            const uint64_t bd = tc::sdesc(b_hi + kk * 256, 128, sbo);
            tc::mma_bf16(tmem, ad, bd, id, acc);
            acc = 1;
            if (split) {
                const uint32_t a_lo = tc::smem_u32(s.t_lo + a_off), b_lo = tc::smem_u32(s.w_lo + b_off);
                tc::mma_bf16(tmem, ad, tc::sdesc(b_lo + kk * 256, 128, sbo), id, 1);
                tc::mma_bf16(tmem, tc::sdesc(a_lo + kk * 256, 128, sbo), bd, id, 1);
            }
        }
        tc::mma_commit(s.bar);
    }
    const bool ok = __syncthreads_and(tc::mbar_wait(s.bar, phase, polls)) != 0;
    if (ok) phase ^= 1u;
    tc::fence_after_sync();
    return ok;
}

}  // namespace

template <bool SPLIT>
__global__ void __launch_bounds__(TILE) k_nn_tc(const DevPot *__restrict__ pot, const float *__restrict__ wpar,
                                                const int *__restrict__ type_count, const int *__restrict__ order,
                                                const float *__restrict__ G, int gstride, float *__restrict__ e_atom,
                                                float *__restrict__ dEdG, DevErr *err, uint32_t polls)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const DevPot &P = *pot;
    const int t = threadIdx.x, warp = t >> 5;
    // tiles per element and the first one of each
    int first[NNP_MAX_TYPES + 1], base[NNP_MAX_TYPES + 1];
    first[0] = 0;
    base[0] = 0;
    for (int T = 0; T < P.ntypes; ++T) {
        const int c = type_count[T];
        first[T + 1] = first[T] + (c + TILE - 1) / TILE;
        base[T + 1] = base[T] + c;
    }
    const int ntiles = first[P.ntypes];
    Smem s0;
    s0.bar = reinterpret_cast<uint64_t *>(smem_raw);
    s0.slot = reinterpret_cast<uint32_t *>(smem_raw + 8);
    if (t == 0) {
        tc::mbar_init(s0.bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tc::tmem_alloc(s0.slot, TMEM_COLS);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *s0.slot;
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    uint32_t phase = 0;
    int staged = -1;
    bool ok = true;
    // The first 64 values of this thread's G row of the next tile are loaded
    // into registers while the current tile computes.
    float4 row[16];
    auto fetch_row = [&](int gg) {
        if (gg >= ntiles) return;
        int Tn = 0;
        while (gg >= first[Tn + 1]) ++Tn;
        const int jn = (gg - first[Tn]) * TILE + t;
        const bool ln = jn < type_count[Tn];
        const float *Gn = G + (ln ? order[base[Tn] + jn] : 0) * (i64)gstride;
#pragma unroll
        for (int q = 0; q < 16; ++q)
            row[q] = (ln && 4 * q + 4 <= gstride) ? *reinterpret_cast<const float4 *>(Gn + 4 * q)
                                                  : make_float4(0.f, 0.f, 0.f, 0.f);
    };
    fetch_row(blockIdx.x);
    for (int g = blockIdx.x; g < ntiles && ok; g += gridDim.x) {
        int T = 0;
        while (g >= first[T + 1]) ++T;
        const DevType &DT = P.t[T];
        TcPlan p;
        make_plan(DT, SPLIT, p);
        const Smem s = carve(smem_raw, p, SPLIT);
        const float *net = wpar + DT.woff;
        const int L = DT.nlayer, nin = DT.nodes[0], nout = DT.nodes[L];
        const float *inpw = net, *inpb = net + nin, *outw = net + 2 * nin, *outb = outw + nout;
        const float *b_out, *w_out;
        int ws_out;
        layer_ptrs(net, DT, L - 1, b_out, w_out, ws_out);
        // ---- weights of this element in the operand layouts (zero padded)
        if (staged != T) {
            __syncthreads();
            for (int h = 0; h + 1 < L; ++h) {
                const int ni = DT.nodes[h], no = DT.nodes[h + 1], Pi = p.P[h], Po = p.P[h + 1];
                const float *bh, *wth;
                int ws;
                layer_ptrs(net, DT, h, bh, wth, ws);
                for (int q = t; q < Po * Pi; q += TILE) {
                    const int n = q / Pi, m = q - n * Pi;       // W[n][m], n < Po (out), m < Pi (in)
                    const float w = (n < no && m < ni) ? wth[m * ws + n] : 0.f;
                    const __nv_bfloat16 hi = __float2bfloat16_rn(w);
                    s.w_hi[p.wf[h] + tc::kmaj(n, m, Pi)] = hi;
                    s.w_hi[p.wb[h] + tc::kmaj(m, n, Po)] = hi;
                    if (SPLIT) {
                        const __nv_bfloat16 lo = __float2bfloat16_rn(w - __bfloat162float(hi));
                        s.w_lo[p.wf[h] + tc::kmaj(n, m, Pi)] = lo;
                        s.w_lo[p.wb[h] + tc::kmaj(m, n, Po)] = lo;
                    }
                }
            }
            // per-element vectors, read by every thread in the epilogues
            {
                float *vb = s.vec + 2 * nin;
                for (int q = t; q < nin; q += TILE) {
                    s.vec[q] = inpw[q];
                    s.vec[nin + q] = inpb[q];
                }
                for (int h = 0; h + 1 < L; ++h) {
                    const float *bh, *wth;
                    int ws;
                    layer_ptrs(net, DT, h, bh, wth, ws);
                    for (int q = t; q < DT.nodes[h + 1]; q += TILE) vb[q] = bh[q];
                    vb += DT.nodes[h + 1];
                }
                for (int q = t; q < DT.nodes[L - 1]; q += TILE) vb[q] = w_out[q * ws_out];
            }
            staged = T;
            __syncthreads();        // the vectors are read below by every thread (A_0 conversion)
        }
        const int neuron = DT.neuron;
        const float cn = DT.c, outw0 = outw[0], eoff = outb[0] + b_out[0] * outw[0];
        const float *v_inpw = s.vec, *v_inpb = s.vec + nin, *v_wout = s.vec + p.vfloats - DT.nodes[L - 1];
        // ---- this thread's atom
        const int j = (g - first[T]) * TILE + t;
        const bool live = j < type_count[T];
        const i64 i = live ? order[base[T] + j] : 0;
        // A_0 = inpw * (G + inpb), zero padded; the row is read as float4
        // (gstride is a multiple of 4 and rows start 16-byte aligned): the
        // first 64 values prefetched during the previous tile, the rest here
        {
#pragma unroll
            for (int k0 = 0; k0 < 64; k0 += 8) {            // from the prefetched registers
                if (k0 < p.P[0]) {
                    const float4 lo4 = row[k0 / 4], hi4 = row[k0 / 4 + 1];
                    const float g8[8] = {lo4.x, lo4.y, lo4.z, lo4.w, hi4.x, hi4.y, hi4.z, hi4.w};
                    float v[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const int k = k0 + q;
                        v[q] = (live && k < nin) ? v_inpw[k] * (g8[q] + v_inpb[k]) : 0.f;
                    }
                    store8(s.t_hi, SPLIT ? s.t_lo : nullptr, p.tile[0] + tc::kmaj(t, k0, p.P[0]), v);
                }
            }
            const float *Gi = G + i * gstride;
#pragma unroll 4
            for (int k0 = 64; k0 < p.P[0]; k0 += 8) {
                float4 lo4 = make_float4(0.f, 0.f, 0.f, 0.f), hi4 = lo4;
                if (live && k0 + 4 <= gstride) lo4 = *reinterpret_cast<const float4 *>(Gi + k0);
                if (live && k0 + 8 <= gstride) hi4 = *reinterpret_cast<const float4 *>(Gi + k0 + 4);
                const float g[8] = {lo4.x, lo4.y, lo4.z, lo4.w, hi4.x, hi4.y, hi4.z, hi4.w};
                float v[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int k = k0 + q;
                    v[q] = (live && k < nin) ? v_inpw[k] * (g[q] + v_inpb[k]) : 0.f;
                }
                store8(s.t_hi, SPLIT ? s.t_lo : nullptr, p.tile[0] + tc::kmaj(t, k0, p.P[0]), v);
            }
        }
        fetch_row(g + gridDim.x);
        // ---- forward through the hidden layers
        float e = 0.f;
        for (int h = 0; h + 1 < L && ok; ++h) {
            const int no = DT.nodes[h + 1], Po = p.P[h + 1];
            ok = gemm(s, p.tile[h], p.wf[h], p.P[h], Po, SPLIT, tmem, phase, polls);
            if (!ok) break;
            const bool last = (h + 2 == L);
            int doff = 0, boff = 2 * nin;
            for (int q = 0; q < h; ++q) {
                doff += TILE * DT.nodes[q + 1];
                boff += DT.nodes[q + 1];
            }
            float *dh = s.d + doff;
            const float *bh = s.vec + boff;
            for (int c0 = 0; c0 < Po; c0 += 32) {
                uint32_t r[4][8];                        // up to 32 columns in flight
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (c0 + 8 * u < Po) tc::tmem_ld8_raw(tmem + lane_base + c0 + 8 * u, r[u]);
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (c0 + 8 * u < Po) tc::tmem_wait_tie(r[u]);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int cb = c0 + 8 * u;
                    if (cb >= Po) break;
                    float out[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const int n = cb + q;
                        out[q] = 0.f;
                        if (n < no) {
                            float a, d;
                            tc_activation(neuron, cn, __uint_as_float(r[u][q]) + bh[n], a, d);
                            dh[n * TILE + t] = d;
                            if (last) {
                                // output layer: e = b + sum_n W[0][n] a_n; D = outw W[0][n] f'(z_n)
                                const float wo = v_wout[n];
                                e = fmaf(wo, a, e);
                                out[q] = outw0 * wo * d;
                            } else {
                                out[q] = a;
                            }
                        }
                    }
                    // next layer's input A_{h+1}, or (last hidden layer) the first
                    // backward operand D_h in region h; both have K = P_{h+1}
                    store8(s.t_hi, SPLIT ? s.t_lo : nullptr, p.tile[last ? h : h + 1] + tc::kmaj(t, cb, Po), out);
                }
            }
            if (last && live) e_atom[i] = eoff + e * outw0;
        }
        if (!ok) break;
        // ---- backward: D_{h-1} = (D_h W_h) * f'(z_{h-1}), dE/dG = (D_0 W_0) * inpw;
        // D_h sits in region h with K = P_{h+1}
        for (int h = L - 2; h >= 0 && ok; --h) {
            const int Pi = p.P[h], Po = p.P[h + 1];
            ok = gemm(s, p.tile[h], p.wb[h], Po, Pi, SPLIT, tmem, phase, polls);
            if (!ok) break;
            if (h > 0) {
                int doff = 0;
                for (int q = 0; q < h - 1; ++q) doff += TILE * DT.nodes[q + 1];
                const float *dprev = s.d + doff;
                const int ni = DT.nodes[h];
                for (int c0 = 0; c0 < Pi; c0 += 32) {
                    uint32_t r[4][8];
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        if (c0 + 8 * u < Pi) tc::tmem_ld8_raw(tmem + lane_base + c0 + 8 * u, r[u]);
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        if (c0 + 8 * u < Pi) tc::tmem_wait_tie(r[u]);
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int cb = c0 + 8 * u;
                        if (cb >= Pi) break;
                        float out[8];
#pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            const int n = cb + q;
                            out[q] = (n < ni) ? __uint_as_float(r[u][q]) * dprev[n * TILE + t] : 0.f;
                        }
                        store8(s.t_hi, SPLIT ? s.t_lo : nullptr, p.tile[h - 1] + tc::kmaj(t, cb, Pi), out);
                    }
                }
            } else {
                // dE/dG row, written as float4 (gstride is a multiple of 4)
                float *o = dEdG + i * gstride;
                for (int c0 = 0; c0 < Pi; c0 += 32) {
                    uint32_t r[4][8];
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        if (c0 + 8 * u < Pi) tc::tmem_ld8_raw(tmem + lane_base + c0 + 8 * u, r[u]);
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        if (c0 + 8 * u < Pi) tc::tmem_wait_tie(r[u]);
                    if (live) {
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            const int cb = c0 + 8 * u;
                            if (cb >= Pi) break;
                            float w[8];
#pragma unroll
                            for (int q = 0; q < 8; ++q) {
                                const int n = cb + q;
                                w[q] = (n < nin) ? __uint_as_float(r[u][q]) * v_inpw[n] : 0.f;
                            }
                            if (cb + 4 <= gstride)
                                *reinterpret_cast<float4 *>(o + cb) = make_float4(w[0], w[1], w[2], w[3]);
                            if (cb + 8 <= gstride)
                                *reinterpret_cast<float4 *>(o + cb + 4) = make_float4(w[4], w[5], w[6], w[7]);
                        }
                    }
                }
            }
        }
    }
    if (!ok && t == 0) atomicMax(&err->nonfinite, 2);
    // every issued MMA chain was waited for unless a wait gave up (in every
    // thread alike); then the chain still in flight is waited for once more,
    // with the full default bound, before the TMEM is released
    if (!ok) tc::mbar_wait(s0.bar, phase, WAIT_POLLS);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, TMEM_COLS);
}

// Shared-memory bytes of the largest element's plan, or 0 when the networks
// do not fit the tensor-core path (output layer wider than one neuron, no
// hidden layer, a layer wider than 128, or shared memory above the CTA limit).
int tc_smem_bytes(const Engine &E, bool split)
{
    int big = 0;
    for (int T = 0; T < E.dpot.ntypes; ++T) {
        const DevType &DT = E.dpot.t[T];
        if (DT.nlayer < 2 || DT.nodes[DT.nlayer] != 1) return 0;
        for (int l = 0; l < DT.nlayer; ++l)
            if (pad16(DT.nodes[l]) > (int)TMEM_COLS) return 0;
        TcPlan p;
        make_plan(DT, split, p);
        big = std::max(big, p.total);
    }
    return big <= 227 * 1024 ? big : 0;
}

std::string run_nn_tc(Engine &E, bool split)
{
    const int64_t N = E.n_atoms;
    if (N == 0) return "";
    const int sm = tc_smem_bytes(E, split);
    if (sm == 0) return "networks do not fit the tensor-core path";
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // at most 4 CTAs per SM: 4 x 128 TMEM columns is the SM's 512
    int per_sm = std::max(1, std::min(4, (228 * 1024) / (sm + 1024)));
    if (E.tune.tc_per_sm > 0) per_sm = std::min(per_sm, E.tune.tc_per_sm);   // autotuned (nnp_tune.cpp)
    const int64_t tiles = (N + TILE - 1) / TILE + E.dpot.ntypes;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)nsm * per_sm));
    const uint32_t polls = E.mma_wait_polls > 0 ? E.mma_wait_polls : WAIT_POLLS;
    if (split) {
        cudaFuncSetAttribute(k_nn_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        k_nn_tc<true><<<grid, TILE, sm, E.stream>>>(E.d_pot, E.wpar.p, E.type_fill.p, E.order.p, E.G.p, E.gstride,
                                                   E.e_atom.p, E.dEdG.p, E.err.p, polls);
    } else {
        cudaFuncSetAttribute(k_nn_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        k_nn_tc<false><<<grid, TILE, sm, E.stream>>>(E.d_pot, E.wpar.p, E.type_fill.p, E.order.p, E.G.p, E.gstride,
                                                    E.e_atom.p, E.dEdG.p, E.err.p, polls);
    }
    E.launches += 1;
    E.mark(3);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? "" : std::string("tensor-core networks: ") + cudaGetErrorString(e);
}

}  // namespace nnp
