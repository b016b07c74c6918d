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
