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
    float *smem = reinterpret_cast<float *>(smem4);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int per = nbr_view_floats(cap, ncut_max, ndamp_max, gstride, true);
    const NbrView v = nbr_view(smem + (size_t)warp * ((per + 3) & ~3), cap, ncut_max, ndamp_max, gstride, true);
    // the force view's per-neighbour gradient arrays hold the relative
    // displacement dv_k = V_i - V_k, and its pair-coefficient area the rate
    // of change of the distance, rr_k = u_k . dv_k (cap <= NNP_MAX_NBR <= 4 NNP_PCH)
    float *rr = v.pc;
    const DevPot &P = *pot;
    for (i64 idx = blockIdx.x * (i64)WARPS + warp; idx < N; idx += (i64)gridDim.x * WARPS) {
        const i64 i = order[idx];
        const int II = type[i];
        const DevType &T = P.t[II];
        const int n = stage_neighbors(v, i, cap, nbr, nbr_cnt, P, T, lane);
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
            for (int f = lane; f < B.n; f += 32) {
                const float2 q = rpar[B.par + f];
                float acc = 0.f;
                for (int k = s0; k < s1; ++k) {
                    float val, der;
                    radial_fd(B.form, v.r[k], q.x, q.y, v.fc[B.cut * cap + k], v.fd[B.cut * cap + k], val, der);
                    acc = fmaf(der, rr[k], acc);
                }
                Ci[B.off_g + f] = acc;
            }
        }
        __syncwarp();
        // angular: dG/deps = dG/dcos dcos + dG/dr_a rr_a + dG/dr_b rr_b with
        // dcos = (u_b . dv_a - cos rr_a)/r_a + (u_a . dv_b - cos rr_b)/r_b
        const int TT = P.ntypes * (P.ntypes + 1) / 2;
        for (int tt = 0; tt < TT; ++tt) {
            const DevBlockA B = T.ba[tt];
            if (B.n == 0) continue;
            int J, K;
            tt_decode(tt, J, K);
            Blk k;
            if (!make_blk(v, J, K, k)) continue;
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
        const int per = nbr_view_floats(E.cap, ncut, ndamp, E.gstride, true);
        const size_t sm = (size_t)WARPS * ((per + 3) & ~3) * sizeof(float);
        if (sm > 227 * 1024) return "neighbour capacity too large for the tangent kernel";
        cudaFuncSetAttribute(k_tangent, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_tangent<<<grid_for(N, WARPS, nsm * 16), WARPS * 32, sm, E.stream>>>(
            N, E.d_pot, E.rpar.p, E.apar.p, E.type.p, E.order.p, E.nbr.p, E.nbr_cnt.p, E.cap, ncut, ndamp, E.gstride,
            E.tvec.p, E.tang.p);
        E.launches += 1;
        std::string msg = cuda_msg("tangent symmetry functions");
        if (!msg.empty()) return msg;
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
