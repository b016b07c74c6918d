// nnp_jit.cpp -- symmetry-function and force kernels specialised at run time
// for the loaded potential.
//
// The prebuilt kernels read every angular function's (lambda, zeta, eta) from
// memory and branch on them per pair.  Here the host writes CUDA source in
// which each GAUSS angular block of the potential is straight-line code: the
// bases 0.5 +- 0.5 cos, their powers as a shared multiply ladder, the damping
// products once per group, and every parameter a literal.  NVRTC compiles it
// for sm_100a when the handle is created; the kernels reuse the per-atom
// skeleton of nnp_device.cuh (symm_body / force_body) through a Blocks policy,
// so only the block arithmetic differs from the prebuilt path.  Blocks of
// other forms fall through to the generic code inside the same kernels.
#include <cuda_runtime.h>
#include <nvrtc.h>

#include <sys/stat.h>
#include <unistd.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <map>
#include <mutex>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "nnp_engine.h"

namespace nnp {

extern const char *const kDeviceHeaderSource;   // nnp_device.cuh, embedded at build time

namespace {

std::string flit(float x)
{
    char b[64];
    std::snprintf(b, sizeof b, "%.9ef", x);
    return b;
}

struct Fn {
    float lf, zeta, ieta2;
    int damp, iz;
};

// emits x_b^n (n >= 1 integer) from a binary ladder, memoised
struct Powers {
    std::ostringstream &os;
    std::set<std::string> done;
    explicit Powers(std::ostringstream &o) : os(o) {}
    std::string ladder(int b, int e)   // x_b^(2^e)
    {
        const std::string name = "x" + std::to_string(b) + "_" + std::to_string(1 << e);
        if (e == 0) return "x" + std::to_string(b);
        if (!done.count(name)) {
            const std::string h = ladder(b, e - 1);
            os << "            const float " << name << " = " << h << " * " << h << ";\n";
            done.insert(name);
        }
        return name;
    }
    std::string pw(int b, int n)
    {
        if (n == 0) return "1.0f";
        std::vector<std::string> terms;
        for (int e = 0; (1 << e) <= n; ++e)
            if (n & (1 << e)) terms.push_back(ladder(b, e));
        if (terms.size() == 1) return terms[0];
        const std::string name = "x" + std::to_string(b) + "p" + std::to_string(n);
        if (!done.count(name)) {
            os << "            const float " << name << " = " << terms[0];
            for (size_t k = 1; k < terms.size(); ++k) os << " * " << terms[k];
            os << ";\n";
            done.insert(name);
        }
        return name;
    }
    // x_b^zeta for any zeta: ladder when integer, exp2/log2 otherwise
    std::string power(int b, float zeta, int iz)
    {
        if (iz >= 0) return pw(b, iz);
        const std::string name = "x" + std::to_string(b) + "r" + std::to_string(done.size());
        os << "            const float " << name << " = (x" << b << " > 0.f) ? exp2f(" << flit(zeta) << " * log2f(x" << b
           << ")) : 0.f;\n";
        done.insert(name);
        return name;
    }
};

std::vector<Fn> block_fns(const Engine &E, const DevBlockA &B)
{
    std::vector<Fn> fs;
    for (int f = 0; f < B.n; ++f) {
        const float4 q = E.apar_host[B.par + f];
        int pk;
        std::memcpy(&pk, &q.w, sizeof pk);
        fs.push_back({q.x, q.y, q.z, pk & 0xff, (pk >> 8) - 1});
    }
    return fs;
}

// common per-pair prologue: geometry, bases, damping factors of the used groups
void pair_prologue(std::ostringstream &os, const std::vector<Fn> &fs, std::vector<float> &bases,
                   std::set<int> &damps, bool force)
{
    os << "            int a, b;\n"
          "            pit_slots(k, it, a, b);\n"
          "            const float4 ua = v.u[a], ub = v.u[b];\n"
          "            const float cs = ua.x * ub.x + ua.y * ub.y + ua.z * ub.z;\n";
    for (const Fn &f : fs) {
        bool seen = false;
        for (float x : bases) seen |= (x == f.lf);
        if (!seen) bases.push_back(f.lf);
        damps.insert(f.damp);
    }
    for (size_t b = 0; b < bases.size(); ++b)
        os << "            const float x" << b << " = fabsf(fmaf(" << flit(bases[b]) << ", cs, 0.5f));\n";
    // damping factors: groups 2m and 2m+1 of a neighbour are one float2 (wix)
    std::set<int> pairs;
    for (int d : damps) pairs.insert(d >> 1);
    for (int m : pairs) {
        const std::string M = std::to_string(m);
        os << "            const float2 wpa" << M << " = reinterpret_cast<const float2 *>(v.w)[" << M
           << " * cap + a], wpb" << M << " = reinterpret_cast<const float2 *>(v.w)[" << M << " * cap + b];\n";
        if (force)
            os << "            const float2 dpa" << M << " = reinterpret_cast<const float2 *>(v.wd)[" << M
               << " * cap + a], dpb" << M << " = reinterpret_cast<const float2 *>(v.wd)[" << M << " * cap + b];\n";
    }
    for (int d : damps) {
        const std::string M = std::to_string(d >> 1), c = (d & 1) ? ".y" : ".x";
        os << "            const float wa" << d << " = wpa" << M << c << ", wb" << d << " = wpb" << M << c << ";\n";
        if (force)
            os << "            const float da" << d << " = dpa" << M << c << ", db" << d << " = dpb" << M << c << ";\n";
        else
            os << "            const float w" << d << " = wa" << d << " * wb" << d << ";\n";
    }
}

int base_of(const std::vector<float> &bases, float lf)
{
    for (size_t b = 0; b < bases.size(); ++b)
        if (bases[b] == lf) return (int)b;
    return 0;
}

// Sums over the warp of the per-lane accumulators s0 .. s(nf-1), stored to
// dst[f] by one lane each.  The list (padded with zeros to a power of two) is
// halved at each shuffle offset: a lane keeps one half and adds its partner's
// copy of that half, so nf values cost about nf shuffles instead of 5 nf; once
// one value is left the remaining offsets are plain butterflies.  The lane's
// offset bits then give the index of the sum it holds.
std::string gen_reduce_store(size_t nf, const std::string &acc, const std::string &dst, bool to_float)
{
    std::ostringstream os;
    size_t p2 = 1;
    while (p2 < nf) p2 <<= 1;
    std::vector<std::string> L;
    for (size_t f = 0; f < p2; ++f) L.push_back(f < nf ? "s" + std::to_string(f) : "(" + acc + ")0");
    std::string idx = "0";
    int dup = 0, tmp = 0;
    for (int o = 16; o >= 1; o >>= 1) {
        const std::string O = std::to_string(o);
        if (L.size() == 1) {
            os << "            " << L[0] << " += __shfl_xor_sync(NNP_FULL, " << L[0] << ", " << O << ");\n";
            dup |= o;
            continue;
        }
        const size_t h = L.size() / 2;
        os << "            const bool hb" << O << " = (lane & " << O << ") != 0;\n";
        std::vector<std::string> N;
        for (size_t i = 0; i < h; ++i) {
            const std::string t = "rs" + std::to_string(tmp++);
            os << "            " << acc << " " << t << " = (hb" << O << " ? " << L[h + i] << " : " << L[i]
               << ") + __shfl_xor_sync(NNP_FULL, hb" << O << " ? " << L[i] << " : " << L[h + i] << ", " << O << ");\n";
            N.push_back(t);
        }
        idx += " + (hb" + O + " ? " + std::to_string(h) + " : 0)";
        L = N;
    }
    os << "            { const int fi = " << idx << ";\n"
       << "              if ((lane & " << dup << ") == 0 && fi < " << nf << ") " << dst << "[fi] = "
       << (to_float ? "(float)" : "") << L[0] << "; }\n";
    return os.str();
}

// Body of one GAUSS block's symmetry functions; written relative to the
// block's first function (Gb), so blocks with equal parameters share it.
std::string gen_symm_body(const Engine &E, const DevBlockA &B)
{
    std::ostringstream os;
    const std::vector<Fn> fs = block_fns(E, B);
    os << "        {\n";
    for (size_t f = 0; f < fs.size(); ++f) os << "            Acc s" << f << " = 0;\n";
    os << "            PairIt it = pit_init(k, lane);\n"
          "#pragma unroll 1\n"
          "            for (int p = lane; p < k.npairs; p += 32, pit_next(k, it)) {\n";
    std::ostringstream body;
    std::vector<float> bases;
    std::set<int> damps;
    pair_prologue(body, fs, bases, damps, false);
    Powers P(body);
    for (size_t f = 0; f < fs.size(); ++f) {
        const std::string x = P.power(base_of(bases, fs[f].lf), fs[f].zeta, fs[f].iz);
        body << "            acc_add(s" << f << ", " << x << ", w" << fs[f].damp << ");\n";
    }
    os << body.str() << "            }\n";
    os << gen_reduce_store(fs.size(), "Acc", "Gb", true);
    os << "            return true;\n        }\n";
    return os.str();
}

// Pair pass of one GAUSS block (see force_pairs_generic), relative to the
// block's first dE/dG (eb); coefficients of pair (g, f) at g s + f - qoff
// (qoff: no generated local may take a parameter's name).
std::string gen_force_body(const Engine &E, const DevBlockA &B)
{
    std::ostringstream os;
    const std::vector<Fn> fs = block_fns(E, B);
    os << "        {\n";
    // dE/dG of the block and the coefficients of x^(zeta-1) in dE/dcos
    for (size_t f = 0; f < fs.size(); ++f) {
        os << "            const float e" << f << " = eb[" << f << "];\n";
        os << "            const float q" << f << " = e" << f << " * " << flit(fs[f].zeta * fs[f].lf) << ";\n";
    }
    os << "            PairIt it = pit_init(k, c0 + lane);\n"
          "#pragma unroll NNP_FORCE_UNROLL\n"
          "            for (int p = c0 + lane; p < c1; p += 32, pit_next(k, it)) {\n";
    std::ostringstream body;
    std::vector<float> bases;
    std::set<int> damps;
    pair_prologue(body, fs, bases, damps, true);
    Powers P(body);
    std::map<int, std::string> sc, sp;   // per damping group
    for (size_t f = 0; f < fs.size(); ++f) {
        const Fn &g = fs[f];
        const int b = base_of(bases, g.lf);
        std::string pz, pm1;
        if (g.iz >= 0) {
            pz = P.pw(b, g.iz);
            pm1 = (g.iz >= 1) ? P.pw(b, g.iz - 1) : "";
        } else {
            pm1 = P.power(b, g.zeta - 1.f, -1);
            pz = "(" + pm1 + " * x" + std::to_string(b) + ")";
        }
        if (!pm1.empty()) sc[g.damp] += (sc[g.damp].empty() ? "" : " + ") + ("q" + std::to_string(f) + " * " + pm1);
        sp[g.damp] += (sp[g.damp].empty() ? "" : " + ") + ("e" + std::to_string(f) + " * " + pz);
    }
    body << "            float hc = 0.f, hra = 0.f, hrb = 0.f;\n";
    for (int d : damps) {
        const std::string c = sc[d].empty() ? "0.f" : sc[d];
        const std::string s = sp[d].empty() ? "0.f" : sp[d];
        body << "            { const float gsc = " << c << ";\n";
        body << "              const float gsp = " << s << ";\n";
        body << "              hc = fmaf(gsc, wa" << d << " * wb" << d << ", hc);\n";
        body << "              hra = fmaf(gsp, da" << d << " * wb" << d << ", hra);\n";
        body << "              hrb = fmaf(gsp, wa" << d << " * db" << d << ", hrb); }\n";
    }
    body << "            pair_coeffs(v.pc, v.pcs, it.g * k.s + it.f - qoff, hc, hra, hrb, cs, ua.w, ub.w);\n";
    os << body.str() << "            }\n            return true;\n        }\n";
    return os.str();
}

// Radial term of one neighbour in the force kernel for a GAUSSIAN block:
// amp = sum_f e_f dG_f/dr with dG_f/dr = exp(-g^2) (-2 eta g fc + fc'),
// g = eta (r - rs), (rs, eta) as literals; relative to the block's first
// dE/dG (eb).
std::string gen_radial_force_body(const Engine &E, const DevBlockR &B)
{
    std::ostringstream os;
    os << "        {\n            float amp = 0.f;\n";
    for (int f = 0; f < B.n; ++f) {
        const float2 q = E.rpar_host[B.par + f];
        os << "            { const float g = " << flit(q.y) << " * (r - " << flit(q.x) << ");\n"
           << "              amp = fmaf(eb[" << f << "], expf(-g * g) * fmaf(" << flit(-2.f * q.y)
           << " * g, fc, fcd), amp); }\n";
    }
    os << "            out = amp;\n            return true;\n        }\n";
    return os.str();
}

// Tangent of one GAUSS block's symmetry functions along the displacement
// field (see tangent_body): per pair dG_f = zeta lf x^(zeta-1) w_a w_b dcos
// + x^zeta (w'_a w_b rr_a + w_a w'_b rr_b), relative to the block's first
// entry of the tangent row (Cb).
std::string gen_tangent_body(const Engine &E, const DevBlockA &B)
{
    std::ostringstream os;
    const std::vector<Fn> fs = block_fns(E, B);
    os << "        {\n";
    for (size_t f = 0; f < fs.size(); ++f) os << "            float s" << f << " = 0.f;\n";
    os << "            PairIt it = pit_init(k, lane);\n"
          "#pragma unroll 1\n"
          "            for (int p = lane; p < k.npairs; p += 32, pit_next(k, it)) {\n";
    std::ostringstream body;
    std::vector<float> bases;
    std::set<int> damps;
    pair_prologue(body, fs, bases, damps, true);
    body << "            const float rra = v.pc[a], rrb = v.pc[b];\n"
            "            const float uba = ub.x * v.gx[a] + ub.y * v.gy[a] + ub.z * v.gz[a];\n"
            "            const float uab = ua.x * v.gx[b] + ua.y * v.gy[b] + ua.z * v.gz[b];\n"
            "            const float dcos = (uba - cs * rra) * ua.w + (uab - cs * rrb) * ub.w;\n";
    for (int d : damps) {
        body << "            const float W" << d << " = wa" << d << " * wb" << d << " * dcos;\n";
        body << "            const float R" << d << " = fmaf(da" << d << " * wb" << d << ", rra, wa" << d << " * db" << d
             << " * rrb);\n";
    }
    Powers P(body);
    for (size_t f = 0; f < fs.size(); ++f) {
        const Fn &g = fs[f];
        const int b = base_of(bases, g.lf);
        std::string pz, pm1;
        if (g.iz >= 0) {
            pz = P.pw(b, g.iz);
            pm1 = (g.iz >= 1) ? P.pw(b, g.iz - 1) : "";
        } else {
            pm1 = P.power(b, g.zeta - 1.f, -1);
            pz = "(" + pm1 + " * x" + std::to_string(b) + ")";
        }
        const std::string d = std::to_string(g.damp);
        body << "            s" << f << " = fmaf(" << pz << ", R" << d << ", s" << f << ");\n";
        if (!pm1.empty())
            body << "            s" << f << " = fmaf(" << pm1 << ", " << flit(g.zeta * g.lf) << " * W" << d << ", s" << f
                 << ");\n";
    }
    os << body.str() << "            }\n";
    os << gen_reduce_store(fs.size(), "float", "Cb", false);
    os << "            return true;\n        }\n";
    return os.str();
}

// switch cases of a dispatcher: keys with the same body share one case
std::string group_cases(const std::vector<std::pair<int, std::string>> &cases)
{
    std::vector<std::string> bodies;
    std::vector<std::vector<int>> keys;
    for (const auto &c : cases) {
        size_t i = 0;
        while (i < bodies.size() && bodies[i] != c.second) ++i;
        if (i == bodies.size()) {
            bodies.push_back(c.second);
            keys.emplace_back();
        }
        keys[i].push_back(c.first);
    }
    std::ostringstream os;
    for (size_t i = 0; i < bodies.size(); ++i) {
        for (int k : keys[i]) os << "        case " << k << ":\n";
        os << bodies[i];
    }
    return os.str();
}

std::string make_source(const Engine &E, const TuneParams &tp)
{
    std::ostringstream os;
    // Launch-bound, unroll and chunk choices, as macros at the top of the
    // source (TuneParams; defaults in nnp_engine.h, replaced by the
    // autotuner).  Resident blocks per SM the compiler budgets registers for
    // (at most 255, 128, 85, 64 registers for 1..4 blocks of NNP_WARPS warps).
    // Measured on the batched workload: 4 blocks make the symmetry-function
    // kernel 3 % faster than 3 (64 instead of 71 registers; its shared memory
    // allows 4); the force kernel is fastest unconstrained (115 registers, 2
    // blocks by its shared memory; capped at 128 registers it is 3 % slower).
    os << "#define NNP_SYMM_MINB " << tp.symm_minb << "\n#define NNP_FORCE_MINB " << tp.force_minb
       << "\n#define NNP_FORCE_UNROLL " << tp.force_unroll << "\n";
    // pairs per chunk of the force kernel; small values split the pair rows
    // between many chunks (used by a test)
    if (tp.force_chunk != NNP_PCH) os << "#define NNP_FORCE_CHUNK " << tp.force_chunk << "\n";
    os << "#include \"nnp_device.cuh\"\nnamespace nnp {\nstruct JitBlocks {\n";
    std::vector<std::pair<int, std::string>> sy, fo, ta, ra;
    const int T = E.dpot.ntypes, TT = T * (T + 1) / 2;
    for (int II = 0; II < T; ++II)
        for (int J = 0; J < T; ++J) {
            const DevBlockR &B = E.dpot.t[II].br[J];
            if (B.n > 0 && B.form == RAD_GAUSSIAN) ra.emplace_back(II * NNP_MAX_TYPES + J, gen_radial_force_body(E, B));
        }
    for (int II = 0; II < T; ++II)
        for (int tt = 0; tt < TT; ++tt) {
            const DevBlockA &B = E.dpot.t[II].ba[tt];
            if (B.n == 0 || B.form != ANG_GAUSS) continue;
            sy.emplace_back(II * NNP_MAX_TT + tt, gen_symm_body(E, B));
            fo.emplace_back(II * NNP_MAX_TT + tt, gen_force_body(E, B));
            ta.emplace_back(II * NNP_MAX_TT + tt, gen_tangent_body(E, B));
        }
    os << "    template <typename Acc>\n"
          "    __device__ static bool symm(const NbrView &v, int II, int tt, const Blk &k, int cap, int lane, float *Gb)\n"
          "    {\n        switch (II * NNP_MAX_TT + tt) {\n"
       << group_cases(sy) << "        default: return false;\n        }\n    }\n";
    os << "    __device__ static bool force(const NbrView &v, int II, int tt, const Blk &k, int c0, int c1, int qoff,\n"
          "                                 int cap, int lane, const float *eb)\n"
          "    {\n        switch (II * NNP_MAX_TT + tt) {\n"
       << group_cases(fo) << "        default: return false;\n        }\n    }\n";
    os << "    __device__ static bool radial_force(int II, int t, float r, float fc, float fcd, const float *eb, float &out)\n"
          "    {\n        switch (II * NNP_MAX_TYPES + t) {\n"
       << group_cases(ra) << "        default: return false;\n        }\n    }\n";
    // radial sums of the symmetry-function kernel with the form fixed per case
    {
        bool used[16] = {};
        for (int II = 0; II < T; ++II)
            for (int J = 0; J < T; ++J) {
                const DevBlockR &B = E.dpot.t[II].br[J];
                if (B.n > 0 && B.form >= 0 && B.form < 16) used[B.form] = true;
            }
        os << "    template <typename Acc>\n"
              "    __device__ static bool radial_symm(int form, const NbrView &v, const float *fcv, float rs, float eta,\n"
              "                                       int k0, int s1, int G, Acc &acc)\n"
              "    {\n        switch (form) {\n";
        for (int f = 0; f < 16; ++f)
            if (used[f])
                os << "        case " << f << ": acc = radial_sum<" << f << ", Acc>(v, fcv, rs, eta, k0, s1, G); return true;\n";
        os << "        default: return false;\n        }\n    }\n";
        os << "    __device__ static bool radial_tangent(int form, const NbrView &v, const float *fcv, const float *fdv,\n"
              "                                          const float *rr, float rs, float eta, int k0, int s1, int G,\n"
              "                                          float &acc)\n"
              "    {\n        switch (form) {\n";
        for (int f = 0; f < 16; ++f)
            if (used[f])
                os << "        case " << f << ": acc = radial_tangent_sum<" << f
                   << ">(v, fcv, fdv, rr, rs, eta, k0, s1, G); return true;\n";
        os << "        default: return false;\n        }\n    }\n";
    }
    os << "    __device__ static bool tangent(const NbrView &v, int II, int tt, const Blk &k, int cap, int lane, float *Cb)\n"
          "    {\n        switch (II * NNP_MAX_TT + tt) {\n"
       << group_cases(ta) << "        default: return false;\n        }\n    }\n};\n}  // namespace nnp\n";
    os << R"(
extern "C" __global__ void __launch_bounds__(NNP_WARPS * 32, NNP_SYMM_MINB)
k_symm_jit(long long N, const nnp::DevPot *__restrict__ pot, const float2 *__restrict__ rpar,
           const float4 *__restrict__ apar, const int *__restrict__ type, const int *__restrict__ order,
           const float4 *__restrict__ nbr,
           const int *__restrict__ nbr_cnt, int cap, int ncut_max, int ndamp_max, int gstride, float *__restrict__ G)
{
    extern __shared__ float4 smem4[];
    nnp::symm_body<float, nnp::JitBlocks>(N, pot, rpar, apar, type, order, nbr, nbr_cnt, cap, ncut_max, ndamp_max, gstride,
                                          G, reinterpret_cast<float *>(smem4));
}

extern "C" __global__ void __launch_bounds__(NNP_WARPS * 32, NNP_FORCE_MINB)
k_force_jit(long long N, const nnp::DevPot *__restrict__ pot, const float2 *__restrict__ rpar,
            const float4 *__restrict__ apar, const int *__restrict__ type, const int *__restrict__ order,
           const float4 *__restrict__ nbr,
            const int *__restrict__ nbr_cnt, int cap, int ncut_max, int ndamp_max, int gstride,
            const float *__restrict__ dEdG, double *__restrict__ F, nnp::DevErr *err,
            const int *__restrict__ atom_struct, double *__restrict__ vir)
{
    extern __shared__ float4 smem4[];
    nnp::force_body<nnp::JitBlocks>(N, pot, rpar, apar, type, order, nbr, nbr_cnt, cap, ncut_max, ndamp_max, gstride, dEdG,
                                    F, err, reinterpret_cast<float *>(smem4), atom_struct, vir);
}

extern "C" __global__ void __launch_bounds__(NNP_WARPS * 32, 1)
k_tangent_jit(long long N, const nnp::DevPot *__restrict__ pot, const float2 *__restrict__ rpar,
              const float4 *__restrict__ apar, const int *__restrict__ type, const int *__restrict__ order,
              const float4 *__restrict__ nbr, const int *__restrict__ nbr_cnt, int cap, int ncut_max, int ndamp_max,
              int gstride, const float4 *__restrict__ V, float *__restrict__ Cout)
{
    extern __shared__ float4 smem4[];
    nnp::tangent_body<nnp::JitBlocks>(N, pot, rpar, apar, type, order, nbr, nbr_cnt, cap, ncut_max, ndamp_max, gstride, V,
                                      Cout, reinterpret_cast<float *>(smem4));
}
)";
    return os.str();
}

}  // namespace

std::string jit_source(const Engine &E, const TuneParams &p) { return make_source(E, p); }

void jit_release(Engine &E)
{
    if (E.jit_module) cudaLibraryUnload((cudaLibrary_t)E.jit_module);
    E.jit_module = nullptr;
    E.jit_symm = E.jit_force = E.jit_tangent = nullptr;
}

std::string &jit_last_log()
{
    static thread_local std::string log;
    return log;
}

// 64-bit FNV-1a of a text: key of the compiled-kernel and tuning caches
uint64_t source_hash(const std::string &s)
{
    uint64_t h = 1469598103934665603ull;
    for (unsigned char c : s) {
        h ^= c;
        h *= 1099511628211ull;
    }
    return h;
}

// Directory of the on-disk caches: NNP_CACHE_DIR, else ~/.cache/nnp_b200
// ("" when neither is known).
std::string cache_dir()
{
    const char *dir = std::getenv("NNP_CACHE_DIR");
    if (dir && dir[0]) return dir;
    if (const char *home = std::getenv("HOME")) return std::string(home) + "/.cache/nnp_b200";
    return "";
}

std::string cache_path(uint64_t h)
{
    const std::string d = cache_dir();
    if (d.empty()) return "";
    char name[64];
    std::snprintf(name, sizeof name, "/%016llx.cubin", (unsigned long long)h);
    return d + name;
}

// Compiles the specialised kernels with the handle's launch choices.
std::string jit_compile(const Engine &E, std::string &source, std::vector<char> &cubin)
{
    return jit_compile_params(E, E.tune, source, cubin);
}

// Compiles the specialised kernels with launch choices tp; cubins are kept
// per process and on disk (cache_dir()) by a hash of the source.  Safe to call
// from several host threads at once.
std::string jit_compile_params(const Engine &E, const TuneParams &tp, std::string &source, std::vector<char> &cubin)
{
    static std::mutex mu;
    static std::map<uint64_t, std::vector<char>> memo;
    source = make_source(E, tp);
    const uint64_t key = source_hash(source + kDeviceHeaderSource);
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = memo.find(key);
        if (it != memo.end()) {
            cubin = it->second;
            return "";
        }
    }
    const std::string path = cache_path(key);
    if (!path.empty()) {
        std::ifstream in(path, std::ios::binary);
        if (in) {
            std::vector<char> buf((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
            if (!buf.empty()) {
                cubin = buf;
                std::lock_guard<std::mutex> lk(mu);
                memo[key] = buf;
                return "";
            }
        }
    }
    nvrtcProgram prog;
    const char *hdr_src[1] = {kDeviceHeaderSource};
    const char *hdr_name[1] = {"nnp_device.cuh"};
    if (nvrtcCreateProgram(&prog, source.c_str(), "nnp_jit.cu", 1, hdr_src, hdr_name) != NVRTC_SUCCESS)
        return "nvrtcCreateProgram failed";
    const char *opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-lineinfo", "--fmad=true",
                          "--ptxas-options=-v"};
    const nvrtcResult rc = nvrtcCompileProgram(prog, 5, opts);
    size_t logn = 0;
    nvrtcGetProgramLogSize(prog, &logn);
    std::string log(logn, '\0');
    if (logn) nvrtcGetProgramLog(prog, &log[0]);
    while (!log.empty() && log.back() == '\0') log.pop_back();   // the size counts the terminator
    if (rc != NVRTC_SUCCESS) {
        nvrtcDestroyProgram(&prog);
        return "run-time compilation failed: " + log.substr(0, 2000);
    }
    jit_last_log() = log;
    size_t n = 0;
    nvrtcGetCUBINSize(prog, &n);
    cubin.resize(n);
    nvrtcGetCUBIN(prog, cubin.data());
    nvrtcDestroyProgram(&prog);
    {
        std::lock_guard<std::mutex> lk(mu);
        memo[key] = cubin;
    }
    if (!path.empty()) {
        const std::string dir = path.substr(0, path.rfind('/'));
        std::string cmd;
        for (size_t k = 1; k <= dir.size(); ++k)
            if (k == dir.size() || dir[k] == '/') mkdir(dir.substr(0, k).c_str(), 0755);
        const std::string tmp = path + ".tmp" + std::to_string((long long)getpid());
        std::ofstream out(tmp, std::ios::binary);
        if (out) {
            out.write(cubin.data(), (std::streamsize)cubin.size());
            out.close();
            std::rename(tmp.c_str(), path.c_str());
        }
    }
    return "";
}

std::string jit_build(Engine &E)
{
    jit_release(E);
    std::vector<char> cubin;
    std::string msg = jit_compile(E, E.jit_source, cubin);
    if (!msg.empty()) return msg;
    cudaLibrary_t lib;
    if (cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0) != cudaSuccess) {
        cudaGetLastError();
        return "cudaLibraryLoadData failed";
    }
    cudaKernel_t ks, kf, kt;
    if (cudaLibraryGetKernel(&ks, lib, "k_symm_jit") != cudaSuccess ||
        cudaLibraryGetKernel(&kf, lib, "k_force_jit") != cudaSuccess ||
        cudaLibraryGetKernel(&kt, lib, "k_tangent_jit") != cudaSuccess) {
        cudaGetLastError();
        cudaLibraryUnload(lib);
        return "run-time kernels not found";
    }
    E.jit_module = (void *)lib;
    E.jit_symm = (void *)ks;
    E.jit_force = (void *)kf;
    E.jit_tangent = (void *)kt;
    if (std::getenv("NNP_JIT_VERBOSE")) {        // registers and local memory of the compiled kernels
        const char *names[3] = {"k_symm_jit", "k_force_jit", "k_tangent_jit"};
        const void *fns[3] = {(const void *)ks, (const void *)kf, (const void *)kt};
        for (int q = 0; q < 3; ++q) {
            cudaFuncAttributes a;
            if (cudaFuncGetAttributes(&a, fns[q]) == cudaSuccess)
                std::fprintf(stderr, "nnp jit: %s %d registers, %zu bytes local memory\n", names[q], a.numRegs,
                             a.localSizeBytes);
            else
                cudaGetLastError();
        }
    }
    return "";
}

std::string jit_launch(void *fn, int grid, int block, size_t smem, cudaStream_t stream, void **args)
{
    const void *k = (const void *)fn;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(cudaGetLastError());
    const cudaError_t r = cudaLaunchKernel(k, dim3(grid), dim3(block), args, smem, stream);
    if (r != cudaSuccess) return std::string("cudaLaunchKernel: ") + cudaGetErrorString(r);
    return "";
}

}  // namespace nnp
