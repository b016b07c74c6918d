// nnp_train.cu -- weight gradient of the energy(+force) training loss.
//
// With per-structure energy factors gE_s = norm_s^2 (E_s - Eref_s) / B and
// per-atom force factors V_i = w_f / (3 N_s B) (F_i - Fref_i), the gradient
// of L = (1/B) sum_s [ 0.5 (norm_s (E_s - Eref_s))^2
//                      + w_f 0.5/(3 N_s) sum_i |F_i - Fref_i|^2 ]
// is, atom by atom (E = sum_i E_i(G_i), F = -dE/dx):
//   dL/dtheta = sum_i [ gE_i dE_i/dtheta - d/dtheta (dE_i/dG_i . C_i) ],
//   C_i = sum_k dG_i/dx_k . V_k        (tangent of G_i along the field V).
// The energy term is NNPTEFR::error_cost_o1's MSE term with its batch average
// (nnptefr.cpp:1292-1347, 996-1000) and NN::Cost::grad (ml/nn.cpp:1747-1805);
// the force term has no reference counterpart.
//
//   k_tangent   warp per atom: C_i from the staged neighbour geometry
//               (the same basis derivatives as the force kernel, contracted
//               with the relative displacements V_i - V_k instead of scattered)
//   k_nn_train  warp per atom: network forward with its tangent along C_i,
//               reverse pass over both, parameter gradients summed per block
//               in shared memory and added to an FP64 global gradient.
#include <cstdlib>

#include "nnp_device.cuh"
#include "nnp_engine.h"

namespace nnp {

#define WARPS NNP_WARPS

__global__ void __launch_bounds__(WARPS * 32, 1)
k_tangent(i64 N, const DevPot *__restrict__ pot, const float2 *__restrict__ rpar, const float4 *__restrict__ apar,
          const int *__restrict__ type, const int *__restrict__ order, const float4 *__restrict__ nbr,
          const int *__restrict__ nbr_cnt, int cap, int ncut_max, int ndamp_max, int gstride,
          const float4 *__restrict__ V, float *__restrict__ Cout)
{
    extern __shared__ float4 smem4[];
    tangent_body<GenericBlocks>(N, pot, rpar, apar, type, order, nbr, nbr_cnt, cap, ncut_max, ndamp_max, gstride, V, Cout,
                                reinterpret_cast<float *>(smem4));
}

// Per-warp work area of k_nn_train, in floats: per layer a, f', f'', the
// tangent pre-activation and activation (5 rows of maxn), the two input rows,
// and six adjoint rows.
__host__ __device__ inline int train_warp_floats(int nlayer, int maxn) { return (5 * nlayer + 8) * maxn; }

__global__ void __launch_bounds__(WARPS * 32)
k_nn_train(i64 N, const DevPot *__restrict__ pot, const float *__restrict__ wpar, i64 wfloats,
           const int *__restrict__ type, const int *__restrict__ order, const float *__restrict__ G,
           const float *__restrict__ C, int gstride, int maxn, int maxl, const float *__restrict__ gE,
           double *__restrict__ grad)
{
    extern __shared__ float smem[];
    const i64 wf4 = (wfloats + 3) & ~(i64)3;
    float *w_s = smem;
    float *g_s = smem + wf4;
    for (i64 k = threadIdx.x; k < wfloats; k += blockDim.x) {
        w_s[k] = wpar[k];
        g_s[k] = 0.f;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *ws = smem + 2 * wf4 + (size_t)warp * train_warp_floats(maxl, maxn);
    float *A = ws, *D = A + maxl * maxn, *D2 = D + maxl * maxn, *ZT = D2 + maxl * maxn, *AT = ZT + maxl * maxn;
    float *ins = AT + maxl * maxn, *inst = ins + maxn;
    float *ab = inst + maxn, *abt = ab + maxn, *zb = abt + maxn, *zbt = zb + maxn, *nab = zbt + maxn,
          *nabt = nab + maxn;
    const DevPot &P = *pot;
    const bool tan = (C != nullptr);
    for (i64 idx = blockIdx.x * (i64)WARPS + warp; idx < N; idx += (i64)gridDim.x * WARPS) {
        const i64 i = order[idx];
        if ((unsigned)type[i] >= (unsigned)P.ntypes) continue;  // type out of range (reported by the call)
        const DevType &T = P.t[type[i]];
        const NetView Vw = net_view(w_s + T.woff, T);
        float *gt = g_s + T.woff;     // gradient accumulators, same layout as the weights
        const int L = T.nlayer, nin = T.nodes[0];
        const float *Gi = G + i * gstride;
        for (int m = lane; m < nin; m += 32) {
            ins[m] = Vw.inpw[m] * (Gi[m] + Vw.inpb[m]);
            inst[m] = tan ? Vw.inpw[m] * C[i * gstride + m] : 0.f;
        }
        __syncwarp();
        // forward, primal and tangent
        for (int l = 0; l < L; ++l) {
            const int ni = T.nodes[l], no = T.nodes[l + 1], s = Vw.ws[l];
            const int neu = (l == L - 1) ? NEU_LINEAR : T.neuron;
            const float *x = (l == 0) ? ins : A + (l - 1) * maxn;
            const float *xt = (l == 0) ? inst : AT + (l - 1) * maxn;
            for (int n = lane; n < no; n += 32) {
                float z = Vw.b[l][n], zt = 0.f;
                const float *wc = Vw.wt[l] + n;
                for (int m = 0; m < ni; ++m) {
                    z = fmaf(wc[m * s], x[m], z);
                    zt = fmaf(wc[m * s], xt[m], zt);
                }
                float a, d, d2;
                activation(neu, T.c, z, a, d, d2);
                A[l * maxn + n] = a;
                D[l * maxn + n] = d;
                D2[l * maxn + n] = d2;
                ZT[l * maxn + n] = zt;
                AT[l * maxn + n] = d * zt;
            }
            __syncwarp();
        }
        // reverse: phi = gE E_i - (dE_i/dG) . C_i = gE out - out'
        const int nout = T.nodes[L];
        const float ge = gE[i];
        for (int n = lane; n < nout; n += 32) {
            ab[n] = ge * Vw.outw[n];
            abt[n] = tan ? -Vw.outw[n] : 0.f;
        }
        __syncwarp();
        float *gb = gt + 2 * nin + 2 * nout;     // this layer's bias gradient (walks the layout)
        float *glb[NNP_MAX_LAYERS];
        for (int l = 0; l < L; ++l) {
            glb[l] = gb;
            gb += T.nodes[l + 1] + (i64)T.nodes[l] * Vw.ws[l];
        }
        for (int l = L - 1; l >= 0; --l) {
            const int ni = T.nodes[l], no = T.nodes[l + 1], s = Vw.ws[l];
            for (int n = lane; n < no; n += 32) {
                const float d = D[l * maxn + n];
                const float zbn = fmaf(ab[n], d, abt[n] * D2[l * maxn + n] * ZT[l * maxn + n]);
                zb[n] = zbn;
                zbt[n] = abt[n] * d;
                atomicAdd(glb[l] + n, zbn);
            }
            __syncwarp();
            const float *x = (l == 0) ? ins : A + (l - 1) * maxn;
            const float *xt = (l == 0) ? inst : AT + (l - 1) * maxn;
            float *gw = glb[l] + no;
            for (int q = lane; q < ni * no; q += 32) {
                const int m = q / no, n = q - m * no;
                const float g = tan ? fmaf(zb[n], x[m], zbt[n] * xt[m]) : zb[n] * x[m];
                atomicAdd(gw + m * s + n, g);
            }
            if (l > 0) {
                for (int m = lane; m < ni; m += 32) {
                    const float *wr = Vw.wt[l] + m * s;
                    float t = 0.f, tt = 0.f;
                    for (int n = 0; n < no; ++n) {
                        t = fmaf(wr[n], zb[n], t);
                        tt = fmaf(wr[n], zbt[n], tt);
                    }
                    nab[m] = t;
                    nabt[m] = tt;
                }
                __syncwarp();
                for (int m = lane; m < ni; m += 32) {
                    ab[m] = nab[m];
                    abt[m] = nabt[m];
                }
            }
            __syncwarp();
        }
    }
    __syncthreads();
    for (i64 k = threadIdx.x; k < wfloats; k += blockDim.x) {
        const float g = g_s[k];
        if (g != 0.f) atomicAdd(grad + k, (double)g);
    }
}

// ---------------------------------------------------------------- tiled weight gradient
//
// k_nn_train_tile: the same gradient as k_nn_train for tiles of TT_ROWS atoms
// of one element.  Lane r of every warp is atom r of the tile; the warps
// split each layer's columns.  Forward (primal and tangent) and reverse are
// small matrix products over the tile in shared memory, arrays column-major
// with row stride TT_LD so that lanes (atoms) and threads walking columns hit
// distinct banks.  The weight gradient of a layer, sum over the tile's atoms
// of zb x^T + zbt xt^T, is one thread per entry; the bias gradient one warp
// sum per column.  Both add into a gradient copy of the element's network in
// shared memory (no atomics: every entry has one owner per phase), which is
// added to the FP64 global gradient when the CTA moves on to another element
// and at its end.
#define TT_ROWS 32
#define TT_LD 33

// floats of one element's network in wpar (the layout of net_view)
__host__ __device__ inline int net_floats(const DevType &T)
{
    int n = 2 * T.nodes[0] + 2 * T.nodes[T.nlayer];
    for (int l = 0; l < T.nlayer; ++l) n += T.nodes[l + 1] + T.nodes[l] * wt_stride(T.nodes[l + 1]);
    return n;
}

struct TrainTileDims {
    int maxw;      // floats of the largest element network, rounded up to 4
    int maxin;     // widest input layer
    int sumout;    // largest sum of layer widths nodes[1..L] of one element
    int maxn;      // widest layer
};

__host__ __device__ inline size_t train_tile_floats(const TrainTileDims &d)
{
    return 2 * (size_t)d.maxw + (size_t)TT_LD * (2 * d.maxin + 5 * d.sumout + 4 * d.maxn);
}

__global__ void __launch_bounds__(WARPS * 32)
k_nn_train_tile(const DevPot *__restrict__ pot, const float *__restrict__ wpar, const int *__restrict__ type_count,
                const int *__restrict__ order, const float *__restrict__ G, const float *__restrict__ C, int gstride,
                const float *__restrict__ gE, double *__restrict__ grad, TrainTileDims dims)
{
    extern __shared__ float smem[];
    const DevPot &P = *pot;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5, r = lane;
    int first[NNP_MAX_TYPES + 1], base[NNP_MAX_TYPES + 1];
    first[0] = 0;
    base[0] = 0;
    for (int T = 0; T < P.ntypes; ++T) {
        const int c = type_count[T];
        first[T + 1] = first[T] + (c + TT_ROWS - 1) / TT_ROWS;
        base[T + 1] = base[T] + c;
    }
    const int ntiles = first[P.ntypes];
    float *w_s = smem, *g_s = smem + dims.maxw;
    float *ins = g_s + dims.maxw, *inst = ins + TT_LD * dims.maxin;
    float *lay = inst + TT_LD * dims.maxin;                   // per layer A, D, D2, ZT, AT [no][TT_LD]
    float *ab = lay + 5 * TT_LD * dims.sumout, *abt = ab + TT_LD * dims.maxn, *nab = abt + TT_LD * dims.maxn,
          *nabt = nab + TT_LD * dims.maxn;
    const bool tan = (C != nullptr);
    int cur = -1, cur_n = 0;
    auto flush = [&]() {                                       // gradient copy -> FP64 global gradient
        __syncthreads();
        double *gd = grad + P.t[cur].woff;
        for (int k = t; k < cur_n; k += blockDim.x) {
            const float g = g_s[k];
            if (g != 0.f) atomicAdd(gd + k, (double)g);
        }
        __syncthreads();
    };
    for (int g = blockIdx.x; g < ntiles; g += gridDim.x) {
        int T = 0;
        while (g >= first[T + 1]) ++T;
        const DevType &DT = P.t[T];
        if (T != cur) {
            if (cur >= 0) flush();
            cur = T;
            cur_n = net_floats(DT);
            for (int k = t; k < cur_n; k += blockDim.x) {
                w_s[k] = wpar[DT.woff + k];
                g_s[k] = 0.f;
            }
            __syncthreads();
        }
        const NetView Vw = net_view(w_s, DT);
        const int L = DT.nlayer, nin = DT.nodes[0], nout = DT.nodes[L];
        const int j0 = (g - first[T]) * TT_ROWS, cnt = type_count[T];
        // inputs, scaled: warp w loads atoms w, w + 8, ..., lanes over the row
        for (int rr = warp; rr < TT_ROWS; rr += WARPS) {
            const bool lv = j0 + rr < cnt;
            const i64 ir = lv ? order[base[T] + j0 + rr] : 0;
            for (int m = lane; m < nin; m += 32) {
                ins[m * TT_LD + rr] = lv ? Vw.inpw[m] * (G[ir * gstride + m] + Vw.inpb[m]) : 0.f;
                inst[m * TT_LD + rr] = (lv && tan) ? Vw.inpw[m] * C[ir * gstride + m] : 0.f;
            }
        }
        __syncthreads();
        const bool live = j0 + r < cnt;
        // forward, primal and tangent; columns n = warp + 8k, four at a time
        float *la = lay;
        for (int l = 0; l < L; ++l) {
            const int ni = DT.nodes[l], no = DT.nodes[l + 1], s = Vw.ws[l];
            const int neu = (l == L - 1) ? NEU_LINEAR : DT.neuron;
            const float *x = (l == 0) ? ins : la - 5 * TT_LD * ni;   // A and AT of the previous layer
            const float *xt = (l == 0) ? inst : la - TT_LD * ni;
            float *A = la, *D = A + TT_LD * no, *D2 = D + TT_LD * no, *ZT = D2 + TT_LD * no, *AT = ZT + TT_LD * no;
            for (int n0 = warp; n0 < no; n0 += 4 * WARPS) {
                float z[4], zt[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int n = n0 + k * WARPS;
                    z[k] = (n < no) ? Vw.b[l][n] : 0.f;
                    zt[k] = 0.f;
                }
                for (int m = 0; m < ni; ++m) {
                    const float xv = x[m * TT_LD + r], xtv = xt[m * TT_LD + r];
                    const float *wr = Vw.wt[l] + m * s;
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const int n = n0 + k * WARPS;
                        const float w = (n < no) ? wr[n] : 0.f;
                        z[k] = fmaf(w, xv, z[k]);
                        zt[k] = fmaf(w, xtv, zt[k]);
                    }
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int n = n0 + k * WARPS;
                    if (n < no) {
                        float a, d, d2;
                        activation(neu, DT.c, z[k], a, d, d2);
                        A[n * TT_LD + r] = a;
                        D[n * TT_LD + r] = d;
                        D2[n * TT_LD + r] = d2;
                        ZT[n * TT_LD + r] = zt[k];
                        AT[n * TT_LD + r] = d * zt[k];
                    }
                }
            }
            la += 5 * TT_LD * no;
            __syncthreads();
        }
        // reverse seeds: phi = gE E_i - (dE_i/dG) . C_i
        {
            const float ge = live ? gE[order[base[T] + j0 + r]] : 0.f;
            for (int n = warp; n < nout; n += WARPS) {
                ab[n * TT_LD + r] = ge * Vw.outw[n];
                abt[n * TT_LD + r] = (live && tan) ? -Vw.outw[n] : 0.f;
            }
        }
        __syncthreads();
        float *gb = g_s + 2 * nin + 2 * nout;                   // this layer's bias gradient (walks the layout)
        float *glb[NNP_MAX_LAYERS];
        for (int l = 0; l < L; ++l) {
            glb[l] = gb;
            gb += DT.nodes[l + 1] + DT.nodes[l] * Vw.ws[l];
        }
        float *cab = ab, *cabt = abt, *cnab = nab, *cnabt = nabt;
        for (int l = L - 1; l >= 0; --l) {
            const int ni = DT.nodes[l], no = DT.nodes[l + 1], s = Vw.ws[l];
            la -= 5 * TT_LD * no;
            const float *D = la + TT_LD * no, *D2 = D + TT_LD * no, *ZT = D2 + TT_LD * no;
            const float *x = (l == 0) ? ins : la - 5 * TT_LD * ni;
            const float *xt = (l == 0) ? inst : la - TT_LD * ni;
            // zb, zbt in place of the adjoint; bias gradient by warp sums
            for (int n = warp; n < no; n += WARPS) {
                const int q = n * TT_LD + r;
                const float d = D[q];
                const float zb = fmaf(cab[q], d, cabt[q] * D2[q] * ZT[q]);
                cabt[q] = cabt[q] * d;
                cab[q] = zb;
                const float sb = warp_sum(zb);
                if (lane == 0) glb[l][n] += sb;
            }
            __syncthreads();
            // weight gradient: entry (m, n) = sum over atoms of zb_n x_m + zbt_n
            // xt_m, a thread per block of 4 inputs x 2 outputs (12 loads per 16
            // FMA; threads of a warp walk the outputs, so the x rows broadcast)
            float *gw = glb[l] + no;
            const int nb2 = (no + 1) >> 1, nblk = ((ni + 3) >> 2) * nb2;
            for (int e = t; e < nblk; e += blockDim.x) {
                const int mb = e / nb2, m0 = 4 * mb, n0 = 2 * (e - mb * nb2);
                const bool n1ok = n0 + 1 < no;
                const float *z0 = cab + n0 * TT_LD, *zt0 = cabt + n0 * TT_LD;
                const float *z1 = n1ok ? z0 + TT_LD : z0, *zt1 = n1ok ? zt0 + TT_LD : zt0;
                const float *xr[4], *xtr[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int m = min(m0 + u, ni - 1);
                    xr[u] = x + m * TT_LD;
                    xtr[u] = xt + m * TT_LD;
                }
                float acc[4][2];
#pragma unroll
                for (int u = 0; u < 4; ++u) acc[u][0] = acc[u][1] = 0.f;
#pragma unroll 4
                for (int a = 0; a < TT_ROWS; ++a) {
                    const float za = z0[a], zta = zt0[a], zb1 = z1[a], ztb = zt1[a];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const float xv = xr[u][a], xtv = xtr[u][a];
                        acc[u][0] = fmaf(za, xv, fmaf(zta, xtv, acc[u][0]));
                        acc[u][1] = fmaf(zb1, xv, fmaf(ztb, xtv, acc[u][1]));
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    if (m0 + u < ni) {
                        gw[(m0 + u) * s + n0] += acc[u][0];
                        if (n1ok) gw[(m0 + u) * s + n0 + 1] += acc[u][1];
                    }
                }
            }
            // adjoint of the layer input: W^T zb
            if (l > 0) {
                for (int m = warp; m < ni; m += WARPS) {
                    const float *wr = Vw.wt[l] + m * s;
                    float a = 0.f, at = 0.f;
                    for (int n = 0; n < no; ++n) {
                        a = fmaf(wr[n], cab[n * TT_LD + r], a);
                        at = fmaf(wr[n], cabt[n * TT_LD + r], at);
                    }
                    cnab[m * TT_LD + r] = a;
                    cnabt[m * TT_LD + r] = at;
                }
            }
            __syncthreads();
            float *s1 = cab, *s2 = cabt;
            cab = cnab;
            cabt = cnabt;
            cnab = s1;
            cnabt = s2;
        }
    }
    if (cur >= 0) flush();
}

static int grid_for(int64_t items, int per_block, int max_blocks)
{
    int64_t b = (items + per_block - 1) / per_block;
    if (b < 1) b = 1;
    if (b > max_blocks) b = max_blocks;
    return (int)b;
}

static std::string cuda_msg(const char *what)
{
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return "";
    return std::string(what) + ": " + cudaGetErrorString(e);
}

std::string run_train_grad(Engine &E, bool with_force)
{
    const int64_t N = E.n_atoms;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaMemsetAsync(E.pgrad.p, 0, sizeof(double) * (size_t)E.wfloats, E.stream) != cudaSuccess)
        return cuda_msg("gradient reset");
    if (N == 0) return "";
    int ncut = E.dpot.ncut > 0 ? E.dpot.ncut : 1, ndamp = 1, maxn = 1, maxl = 1;
    for (int t = 0; t < E.dpot.ntypes; ++t) {
        ndamp = std::max(ndamp, E.dpot.t[t].ndamp);
        maxl = std::max(maxl, E.dpot.t[t].nlayer);
        for (int l = 0; l <= E.dpot.t[t].nlayer; ++l) maxn = std::max(maxn, E.dpot.t[t].nodes[l]);
    }
    maxn = (maxn + 3) & ~3;
    if (with_force) {
        const int per = nbr_view_floats(E.cap, ncut, ndamp, E.gstride, true,
                                        (E.use_jit && E.jit_tangent) ? E.tune.force_chunk : NNP_PCH);
        const size_t sm = (size_t)WARPS * ((per + 3) & ~3) * sizeof(float);
        if (sm > 227 * 1024) return "neighbour capacity too large for the tangent kernel";
        const int grid = grid_for(N, WARPS, nsm * 16);
        E.launches += 1;
        if (E.use_jit && E.jit_tangent) {
            long long n = N;
            int cap = E.cap, gs = E.gstride;
            void *args[] = {&n, &E.d_pot, &E.rpar.p, &E.apar.p, &E.type.p, &E.order.p, &E.nbr.p, &E.nbr_cnt.p,
                            &cap, &ncut, &ndamp, &gs, &E.tvec.p, &E.tang.p};
            std::string msg = jit_launch(E.jit_tangent, grid, WARPS * 32, sm, E.stream, args);
            if (!msg.empty()) return msg;
        } else {
            cudaFuncSetAttribute(k_tangent, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k_tangent<<<grid, WARPS * 32, sm, E.stream>>>(N, E.d_pot, E.rpar.p, E.apar.p, E.type.p, E.order.p, E.nbr.p,
                                                          E.nbr_cnt.p, E.cap, ncut, ndamp, E.gstride, E.tvec.p, E.tang.p);
            std::string msg = cuda_msg("tangent symmetry functions");
            if (!msg.empty()) return msg;
        }
    }
    // tiles of one element's atoms when their arrays fit in shared memory
    // (NNP_TRAIN_TILE=0 selects the warp-per-atom kernel)
    TrainTileDims dims{1, 1, 1, 1};
    for (int t = 0; t < E.dpot.ntypes; ++t) {
        const DevType &T = E.dpot.t[t];
        int so = 0;
        for (int l = 0; l < T.nlayer; ++l) so += T.nodes[l + 1];
        dims.maxw = std::max(dims.maxw, (net_floats(T) + 3) & ~3);
        dims.maxin = std::max(dims.maxin, T.nodes[0]);
        dims.sumout = std::max(dims.sumout, so);
        for (int l = 0; l <= T.nlayer; ++l) dims.maxn = std::max(dims.maxn, T.nodes[l]);
    }
    const size_t smt = train_tile_floats(dims) * sizeof(float);
    const char *tile_env = std::getenv("NNP_TRAIN_TILE");
    if (smt <= 227 * 1024 && !(tile_env && tile_env[0] == '0')) {
        cudaFuncSetAttribute(k_nn_train_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smt);
        const int per_sm = std::max(1, std::min(4, (int)((228 * 1024) / (smt + 1024))));
        const int grid = grid_for(N / TT_ROWS + E.dpot.ntypes, 1, nsm * per_sm);
        k_nn_train_tile<<<grid, WARPS * 32, smt, E.stream>>>(E.d_pot, E.wpar.p, E.type_fill.p, E.order.p, E.G.p,
                                                            with_force ? E.tang.p : nullptr, E.gstride, E.gE.p,
                                                            E.pgrad.p, dims);
        E.launches += 1;
        return cuda_msg("k_nn_train_tile");
    }
    const size_t sm = (size_t)(2 * ((E.wfloats + 3) & ~3) + WARPS * train_warp_floats(maxl, maxn)) * sizeof(float);
    if (sm > 227 * 1024) return "networks too large for the shared-memory training kernel";
    cudaFuncSetAttribute(k_nn_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_nn_train<<<grid_for(N, WARPS * 16, nsm * 2), WARPS * 32, sm, E.stream>>>(
        N, E.d_pot, E.wpar.p, E.wfloats, E.type.p, E.order.p, E.G.p, with_force ? E.tang.p : nullptr, E.gstride, maxn,
        maxl, E.gE.p, E.pgrad.p);
    E.launches += 1;
    return cuda_msg("network gradients");
}

}  // namespace nnp

namespace nnp {

// One ADAM step (opt::algo::ADAM::step, opt/algo.cpp:280-296) over the n
// network parameters, with the gradient of the last training call still on
// the device (grad, wpar layout, at idx[i]): running averages m, v of the
// gradient and its square, p -= gamma b1ii m / (sqrt(b2ii v) + eps) on the
// FP64 master copy p64, and its FP32 value written into the networks' table.
// After the step, nnptefr's weight decay (nnptefr.cpp:1034-1057) of kind reg
// (0 LASSO sgn(p), 1 RIDGE p, 2 HUBER p / sqrt(1 + p^2), 3 ASINH asinh(p),
// anything else none) with strength gamma * eta on the weights (wmask 1; the
// biases have 0), evaluated at the parameters before the step.
__global__ void k_adam(int64_t n, const int64_t *__restrict__ idx, const double *__restrict__ grad,
                       double *__restrict__ p64, double *__restrict__ m, double *__restrict__ v,
                       float *__restrict__ wpar, double gamma, double b1ii, double b2ii, double eps,
                       const unsigned char *__restrict__ wmask, int reg, double eta)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    constexpr double beta1 = 0.9, beta2 = 0.999;
    const double g = grad[idx[i]];
    double mm = m[i], vv = v[i];
    mm *= beta1;
    mm += (1.0 - beta1) * g;
    vv *= beta2;
    vv += (1.0 - beta2) * g * g;
    m[i] = mm;
    v[i] = vv;
    const double po = p64[i];
    double p = po - gamma * b1ii * mm / (sqrt(b2ii * vv) + eps);
    if (reg >= 0 && reg <= 3 && wmask[i]) {
        const double f = reg == 0 ? (double)((po > 0) - (po < 0))
                         : reg == 1 ? po
                         : reg == 2 ? po / sqrt(1.0 + po * po)
                                    : asinh(po);
        p -= gamma * eta * f;
    }
    p64[i] = p;
    wpar[idx[i]] = (float)p;
}

std::string run_adam(Engine &E, double gamma, double eps, int reg, double eta)
{
    const int64_t n = (int64_t)E.adam_idx_host.size();
    if (n == 0) return "";
    const double b1ii = 1.0 / (1.0 - E.adam_b1i), b2ii = 1.0 / (1.0 - E.adam_b2i);
    k_adam<<<(int)((n + 255) / 256), 256, 0, E.stream>>>(n, E.adam_idx.p, E.pgrad.p, E.adam_p.p, E.adam_m.p,
                                                           E.adam_v.p, E.wpar.p, gamma, b1ii, b2ii, eps,
                                                           E.adam_wmask.p, reg, eta);
    E.launches += 1;
    E.adam_b1i *= 0.9;
    E.adam_b2i *= 0.999;
    return cuda_msg("ADAM step");
}

}  // namespace nnp

namespace nnp {

namespace {

// nnptefr's normalisation of a structure's energy error (nnptefr.cpp:614-620)
__device__ inline double norm_factor(int mode, double nat)
{
    switch (mode) {
    case 1: return 1.0 / nat;
    case 2: return 1.0 / sqrt(nat);
    case 3: return 1.0 / cbrt(nat);
    case 4: return 1.0 / (log(nat) + 1.0);
    default: return 1.0;
    }
}

// One block per structure: the energy term of NNPTEFR::error_cost_o1
// (nnptefr.cpp:1331-1380: dU = norm (E - E_ref), the loss of kind loss_kind
// and its factor gf = norm dloss/ddU) and the force term
// 0.5 w_f / (3 N) sum |F - F_ref|^2; writes every atom's energy factor
// gE = gf / B and force adjoint V = w_f (F - F_ref) / (3 N B), and the
// structure's loss / B into part[s].
__global__ void k_train_loss(const int64_t *__restrict__ off, const double *__restrict__ E,
                             const double *__restrict__ e_ref, const double *__restrict__ F,
                             const double *__restrict__ f_ref, double w_f, int norm_mode, int loss_kind, double delta,
                             double bi, float *__restrict__ ge, float4 *__restrict__ tv, double *__restrict__ part)
{
    __shared__ double red[256];
    const int s = blockIdx.x;
    const int64_t a0 = off[s], a1 = off[s + 1];
    const double nat = (double)(a1 - a0);
    const double nrm = norm_factor(norm_mode, nat);
    const double dU = (E[s] - e_ref[s]) * nrm;
    double le, dl;
    switch (loss_kind) {
    case 2: le = fabs(dU); dl = (dU > 0) - (dU < 0); break;
    case 3: { const double a = dU / delta, sq = sqrt(1.0 + a * a); le = delta * delta * (sq - 1.0); dl = dU / sq; } break;
    case 4: {
        const double a = dU / delta, sq = sqrt(1.0 + a * a), lg = log(a + sq);
        le = delta * delta * (1.0 - sq + a * lg);
        dl = lg * delta;
    } break;
    default: le = 0.5 * dU * dU; dl = dU; break;
    }
    const float gf = (float)(nrm * dl * bi);
    const double fs = nat > 0 ? w_f / (3.0 * nat) : 0.0;
    double lf = 0.0;
    for (int64_t a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
        ge[a] = gf;
        if (w_f != 0.0) {
            const double d0 = F[3 * a] - f_ref[3 * a], d1 = F[3 * a + 1] - f_ref[3 * a + 1],
                         d2 = F[3 * a + 2] - f_ref[3 * a + 2];
            lf += d0 * d0 + d1 * d1 + d2 * d2;
            tv[a] = make_float4((float)(fs * d0 * bi), (float)(fs * d1 * bi), (float)(fs * d2 * bi), 0.f);
        }
    }
    red[threadIdx.x] = lf;
    __syncthreads();
    for (int k = blockDim.x / 2; k; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[s] = bi * (le + 0.5 * fs * red[0]);
}

// sum of part[0..S) in a fixed order (one block)
__global__ void k_sum_fixed(int S, const double *__restrict__ part, double *__restrict__ out)
{
    __shared__ double red[256];
    double v = 0.0;
    for (int s = threadIdx.x; s < S; s += blockDim.x) v += part[s];
    red[threadIdx.x] = v;
    __syncthreads();
    for (int k = blockDim.x / 2; k; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// gradient from the networks' table layout into the reference packing
__global__ void k_gather_grad(int64_t n, const int64_t *__restrict__ idx, const double *__restrict__ g,
                              double *__restrict__ out)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = g[idx[i]];
}

}  // namespace

std::string run_train_loss(Engine &E, const int64_t *off, const double *e_ref, const double *f_ref, double w_f,
                           int norm_mode, double *loss_dev)
{
    const int S = E.n_struct;
    const double bi = 1.0 / S;
    k_train_loss<<<S, 256, 0, E.stream>>>(off, E.e_struct.p, e_ref, E.force.p, f_ref, w_f, norm_mode, E.loss_kind,
                                          E.loss_delta, bi, E.gE.p, E.tvec.p, E.loss_part.p);
    k_sum_fixed<<<1, 256, 0, E.stream>>>(S, E.loss_part.p, loss_dev);
    E.launches += 2;
    return cuda_msg("training loss");
}

std::string run_gather_grad(Engine &E, const int64_t *idx, int64_t n, double *out)
{
    if (n == 0) return "";
    k_gather_grad<<<(int)((n + 255) / 256), 256, 0, E.stream>>>(n, idx, E.pgrad.p, out);
    E.launches += 1;
    return cuda_msg("gradient gather");
}

}  // namespace nnp
