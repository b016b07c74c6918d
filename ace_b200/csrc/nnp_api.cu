// nnp_api.cu -- the C ABI of libnnp_b200.so (declared in include/nnp_b200.h).
//
// A handle holds a parsed potential (host copy, for writing it back and for
// parameter get/set), its device form, one stream and the scratch buffers.
// No entry point throws: errors come back as NNP_ERR_* codes with a message.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/nnp_b200.h"
#include "nnp_engine.h"

struct nnp_handle {
    nnp::Engine E;
};

namespace {

thread_local std::string g_create_error;

int fail(nnp_handle *h, int code, const std::string &msg)
{
    if (h) h->E.last_error = msg;
    else g_create_error = msg;
    return code;
}

bool read_file(const char *path, std::string &out)
{
    std::ifstream f(path, std::ios::in | std::ios::binary);
    if (!f) return false;
    std::ostringstream ss;
    ss << f.rdbuf();
    out = ss.str();
    return true;
}

bool is_pinned_or_device(const void *p, bool *device)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        *device = false;
        return false;
    }
    *device = (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged);
    return a.type == cudaMemoryTypeHost || *device;
}

int opt_adam_impl(nnp_handle *h, double gamma, double eps, int reg, double eta);

// After device optimiser steps the parameters live in the device's FP64
// master copy; copy them into the host model before it is read or re-uploaded.
std::string host_params(nnp::Engine &E)
{
    if (!E.host_stale) return "";
    std::vector<double> val(E.adam_idx_host.size());
    cudaError_t ce = cudaMemcpyAsync(val.data(), E.adam_p.p, sizeof(double) * val.size(), cudaMemcpyDeviceToHost, E.stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(E.stream);
    if (ce != cudaSuccess) return std::string("parameter copy failed: ") + cudaGetErrorString(ce);
    size_t k = 0;
    for (auto &net : E.host.nets) {
        const int nl = (int)net.nodes.size() - 1;
        for (int l = 0; l < nl; ++l)
            for (auto &v : net.b[l]) v = val[k++];
        for (int l = 0; l < nl; ++l) {
            const int ni = net.nodes[l], no = net.nodes[l + 1];
            for (int m = 0; m < ni; ++m)
                for (int n = 0; n < no; ++n) net.w[l][(size_t)n * ni + m] = val[k++];
        }
    }
    for (size_t i = 0; i < E.adam_idx_host.size(); ++i) E.wpar_host[E.adam_idx_host[i]] = (float)val[i];
    E.host_stale = false;
    return "";
}

// wpar offset of every network parameter in the reference packing (per type
// in index order: biases by layer, then the weights column-major,
// nn.cpp:881-915), and whether it is a weight
void pack_offsets(const nnp::Engine &E, std::vector<int64_t> &idx, std::vector<unsigned char> *is_weight)
{
    idx.clear();
    if (is_weight) is_weight->clear();
    for (int t = 0; t < E.dpot.ntypes; ++t) {
        const nnp::DevType &T = E.dpot.t[t];
        const int nin = T.nodes[0], nout = T.nodes[T.nlayer];
        int64_t off = T.woff + 2 * nin + 2 * nout;
        std::vector<int64_t> boff(T.nlayer), woff(T.nlayer);
        for (int l = 0; l < T.nlayer; ++l) {
            boff[l] = off;
            woff[l] = off + T.nodes[l + 1];
            off = woff[l] + (int64_t)T.nodes[l] * nnp::wt_stride(T.nodes[l + 1]);
        }
        for (int l = 0; l < T.nlayer; ++l)
            for (int n = 0; n < T.nodes[l + 1]; ++n) {
                idx.push_back(boff[l] + n);
                if (is_weight) is_weight->push_back(0);
            }
        for (int l = 0; l < T.nlayer; ++l) {
            const int ni = T.nodes[l], no = T.nodes[l + 1], st = nnp::wt_stride(no);
            for (int m = 0; m < ni; ++m)
                for (int n = 0; n < no; ++n) {
                    idx.push_back(woff[l] + (int64_t)m * st + n);
                    if (is_weight) is_weight->push_back(1);
                }
        }
    }
}
}  // namespace

namespace nnp {

void Engine::free_all()
{
    rpar.release(); apar.release(); wpar.release(); vac.release();
    rpar64.release(); apar64.release(); cut64.release();
    atom_off.release(); pos.release(); cell.release(); xw.release();
    type.release(); atom_struct.release(); atom_cell.release(); grid.release(); bbox.release();
    cell_cnt.release(); cell_start.release(); cell_fill.release(); cell_atoms.release(); scan_tmp.release();
    cell_tcnt.release();
    cell_pos.release(); order.release(); type_fill.release(); neigh_items.release();
    nbr.release(); nbr_cnt.release(); G.release(); dEdG.release(); e_atom.release();
    e_struct.release(); force.release(); symm_d.release(); err.release(); vir.release(); eatom_d.release();
    tvec.release(); gE.release(); tang.release(); pgrad.release();
    adam_idx.release(); adam_p.release(); adam_m.release(); adam_v.release(); adam_wmask.release();
    loss_part.release(); train_ref.release(); grad_pack.release(); pack_idx.release();
    graph_release();
    jit_release(*this);
    if (d_pot) cudaFree(d_pot);
    d_pot = nullptr;
    if (h_err) cudaFreeHost(h_err);
    h_err = nullptr;
    if (h_stage) cudaFreeHost(h_stage);
    h_stage = nullptr;
    h_stage_bytes = 0;
    if (own_stream && stream) cudaStreamDestroy(stream);
    stream = nullptr;
    own_stream = false;
    for (auto &e : ev)
        if (e) cudaEventDestroy(e);
    for (auto &e : ev) e = nullptr;
}

void Engine::graph_release()
{
    if (graph_exec) cudaGraphExecDestroy((cudaGraphExec_t)graph_exec);
    graph_exec = nullptr;
    graph_key.clear();
    graph_launches = 0;
}

// Build the device potential.  Angular functions of one BasisA that form a
// run of equal eta (BasisA::init, basis_angular.cpp:178-205) share the run's
// first eta for their damping factor, as the reference does.
std::string Engine::build_tables()
{
    const HostPot &H = host;
    const int T = H.ntypes();
    DevPot d;
    std::memset(&d, 0, sizeof d);
    d.ntypes = T;
    d.rc = (float)H.rc;
    d.rc_d = H.rc;
    std::vector<std::pair<int, double>> cuts;
    auto cut_id = [&](int name, double rc) -> int {
        for (size_t k = 0; k < cuts.size(); ++k)
            if (cuts[k].first == name && cuts[k].second == rc) return (int)k;
        if ((int)cuts.size() >= NNP_MAX_CUT) return -1;
        cuts.push_back({name, rc});
        return (int)cuts.size() - 1;
    };
    std::vector<float2> rp;
    std::vector<float4> ap;
    std::vector<double2> rp64;
    std::vector<double4> ap64;
    std::vector<float> wp;
    std::vector<double> vc(T);
    for (int II = 0; II < T; ++II) {
        DevType &t = d.t[II];
        t.n_input = H.n_input(II);
        t.n_input_r = H.n_input_r(II);
        int off = 0;
        for (int J = 0; J < T; ++J) {
            const HostBasisR &b = H.br[II][J];
            const int n = (int)b.rs.size();
            if (n > NNP_MAX_RFUNC) return "a radial basis has more functions than the device path supports";
            const int c = cut_id(b.cut, b.rc);
            if (c < 0) return "too many distinct cutoffs in the potential";
            t.br[J] = {n, off, b.form, c, (int)rp.size()};
            for (int f = 0; f < n; ++f) {
                rp.push_back(make_float2((float)b.rs[f], (float)b.eta[f]));
                rp64.push_back(make_double2(b.rs[f], b.eta[f]));
            }
            off += n;
        }
        int offa = t.n_input_r;
        t.ndamp = 0;
        const int TT = T * (T + 1) / 2;
        for (int tt = 0; tt < TT; ++tt) {
            const HostBasisA &b = H.ba[II][tt];
            const int n = (int)b.eta.size();
            if (n > NNP_MAX_AFUNC) return "an angular basis has more functions than the device path supports";
            const int c = cut_id(b.cut, b.rc);
            if (c < 0) return "too many distinct cutoffs in the potential";
            int int_zeta = 1;
            double etar = n ? b.eta[0] : 0.0;
            for (int f = 0; f < n; ++f) {
                if (f > 0 && std::fabs(b.eta[f] - b.eta[f - 1]) >= 1.0e-6) etar = b.eta[f];
                const double a = 1.0 / (etar * etar);
                int dmp = 0;
                if (b.form == ANG_GAUSS) {
                    dmp = -1;
                    for (int k = 0; k < t.ndamp; ++k)
                        if (t.damp_cut[k] == c && t.damp_a[k] == (float)a) dmp = k;
                    if (dmp < 0) {
                        if (t.ndamp >= NNP_MAX_DAMP) return "too many distinct angular widths for one element";
                        t.damp_cut[t.ndamp] = c;
                        t.damp_a[t.ndamp] = (float)a;
                        dmp = t.ndamp++;
                    }
                }
                const double z = b.zeta[f];
                const int iz = (z == std::floor(z) && z >= 0.0 && z <= 64.0) ? (int)z : -1;
                if (iz < 0) int_zeta = 0;
                const int pk = dmp | ((iz + 1) << 8);
                float w;
                std::memcpy(&w, &pk, sizeof w);
                ap.push_back(make_float4((float)(0.5 * b.lambda[f]), (float)z, (float)a, w));
                ap64.push_back(make_double4(0.5 * b.lambda[f], z, a, 0.0));
            }
            t.ba[tt] = {n, offa, b.form, c, (int)ap.size() - n, int_zeta};
            offa += n;
        }
        // network
        const HostNet &net = H.nets[II];
        t.nlayer = (int)net.nodes.size() - 1;
        if (t.nlayer > NNP_MAX_LAYERS) return "network has more layers than the device path supports";
        for (size_t l = 0; l < net.nodes.size(); ++l) {
            if (net.nodes[l] > NNP_MAX_NODES) return "network layer wider than the device path supports";
            t.nodes[l] = net.nodes[l];
        }
        t.neuron = net.neuron;
        t.c = (float)net.c;
        t.woff = (int64_t)wp.size();
        for (double x : net.inpw) wp.push_back((float)x);
        for (double x : net.inpb) wp.push_back((float)x);
        for (double x : net.outw) wp.push_back((float)x);
        for (double x : net.outb) wp.push_back((float)x);
        for (int l = 0; l < t.nlayer; ++l) {
            const int ni = net.nodes[l], no = net.nodes[l + 1], s = wt_stride(no);
            for (int n = 0; n < no; ++n) wp.push_back((float)net.b[l][n]);
            const size_t base = wp.size();
            wp.resize(base + (size_t)ni * s, 0.f);
            for (int n = 0; n < no; ++n)
                for (int m = 0; m < ni; ++m) wp[base + (size_t)m * s + n] = (float)net.w[l][(size_t)n * ni + m];
        }
        vc[II] = H.types[II].energy;
    }
    d.ncut = (int)cuts.size();
    for (size_t k = 0; k < cuts.size(); ++k) {
        d.cut[k].name = cuts[k].first;
        d.cut[k].rc = (float)cuts[k].second;
        d.cut[k].rci = (float)(1.0 / cuts[k].second);
        d.cut[k].pirci = (float)(3.141592653589793 / cuts[k].second);
    }
    int gs = 1;
    for (int II = 0; II < T; ++II) gs = std::max(gs, d.t[II].n_input);
    gstride = (gs + 3) & ~3;
    wfloats = (int64_t)wp.size();
    rpar_host = rp;
    apar_host = ap;
    rpar64_host = rp64;
    apar64_host = ap64;
    cut64_host.clear();
    for (const auto &c : cuts) cut64_host.push_back(c.second);
    wpar_host = wp;
    vac_host = vc;
    dpot = d;
    return "";
}

std::string Engine::upload()
{
    std::string msg = build_tables();
    if (!msg.empty()) return msg;
    adam_master_stale = true;
    const DevPot &d = dpot;
    std::vector<float2> rp = rpar_host;
    std::vector<float4> ap = apar_host;
    const std::vector<float> &wp = wpar_host;
    const std::vector<double> &vc = vac_host;
    if (rp.empty()) rp.push_back(make_float2(0.f, 0.f));
    if (ap.empty()) ap.push_back(make_float4(0.f, 0.f, 0.f, 0.f));
    std::vector<double2> rp64 = rpar64_host;
    std::vector<double4> ap64 = apar64_host;
    std::vector<double> c64 = cut64_host;
    if (rp64.empty()) rp64.push_back(make_double2(0.0, 0.0));
    if (ap64.empty()) ap64.push_back(make_double4(0.0, 0.0, 0.0, 0.0));
    if (c64.empty()) c64.push_back(0.0);
    cudaError_t e = cudaSuccess;
    auto r = [&](cudaError_t x) { if (x != cudaSuccess && e == cudaSuccess) e = x; };
    if (!d_pot) r(cudaMalloc((void **)&d_pot, sizeof(DevPot)));
    r(rpar.reserve(rp.size()));
    r(apar.reserve(ap.size()));
    r(wpar.reserve(wp.size()));
    r(vac.reserve(vc.size()));
    r(rpar64.reserve(rp64.size()));
    r(apar64.reserve(ap64.size()));
    r(cut64.reserve(c64.size()));
    if (e != cudaSuccess) return std::string("device allocation failed: ") + cudaGetErrorString(e);
    r(cudaMemcpy(d_pot, &d, sizeof d, cudaMemcpyHostToDevice));
    r(cudaMemcpy(rpar.p, rp.data(), rp.size() * sizeof(float2), cudaMemcpyHostToDevice));
    r(cudaMemcpy(apar.p, ap.data(), ap.size() * sizeof(float4), cudaMemcpyHostToDevice));
    r(cudaMemcpy(wpar.p, wp.data(), wp.size() * sizeof(float), cudaMemcpyHostToDevice));
    r(cudaMemcpy(vac.p, vc.data(), vc.size() * sizeof(double), cudaMemcpyHostToDevice));
    r(cudaMemcpy(rpar64.p, rp64.data(), rp64.size() * sizeof(double2), cudaMemcpyHostToDevice));
    r(cudaMemcpy(apar64.p, ap64.data(), ap64.size() * sizeof(double4), cudaMemcpyHostToDevice));
    r(cudaMemcpy(cut64.p, c64.data(), c64.size() * sizeof(double), cudaMemcpyHostToDevice));
    if (e != cudaSuccess) return std::string("potential upload failed: ") + cudaGetErrorString(e);
    return "";
}

}  // namespace nnp

namespace {

int finish_create(nnp_handle *h, nnp_handle **out)
{
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) {
        cudaGetLastError();
        delete h;
        return fail(nullptr, NNP_ERR_CUDA, "no CUDA device available: the NNP path runs only on the GPU");
    }
    nnp::Engine &E = h->E;
    if (cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return fail(nullptr, NNP_ERR_CUDA, "cudaStreamCreate failed");
    }
    E.own_stream = true;
    if (cudaMallocHost((void **)&E.h_err, sizeof(nnp::DevErr)) != cudaSuccess) {
        E.free_all();
        delete h;
        return fail(nullptr, NNP_ERR_CUDA, "cudaMallocHost failed");
    }
    std::string msg = E.upload();
    if (!msg.empty()) {
        E.free_all();
        delete h;
        return fail(nullptr, NNP_ERR_CUDA, msg);
    }
    E.cap = 64;
    // kernels specialised for this basis; NNP_JIT=0 in the environment keeps
    // the prebuilt kernels (a failed compilation does too, and is recorded)
    const char *env = std::getenv("NNP_JIT");
    E.use_jit = !(env && env[0] == '0');
    nnp::tune_from_env(E.tune);
    const char *at = std::getenv("NNP_AUTOTUNE");
    E.autotune = at && at[0] == '1';
    if (E.use_jit) {
        E.jit_error = nnp::jit_build(E);
        if (!E.jit_error.empty()) E.use_jit = false;
    }
    *out = h;
    return NNP_OK;
}

// pinned staging: copy host data through the handle's pinned buffer unless
// it is already pinned (or device) memory
int stage_bytes(nnp::Engine &E, size_t bytes)
{
    if (bytes <= E.h_stage_bytes) return NNP_OK;
    if (E.h_stage) cudaFreeHost(E.h_stage);
    E.h_stage = nullptr;
    E.h_stage_bytes = 0;
    const size_t want = bytes + bytes / 4 + 4096;
    if (cudaMallocHost(&E.h_stage, want) != cudaSuccess) return NNP_ERR_CUDA;
    E.h_stage_bytes = want;
    return NNP_OK;
}

cudaError_t h2d(nnp::Engine &E, void *dst, const void *src, size_t bytes, size_t &stage_off)
{
    if (!bytes) return cudaSuccess;
    bool dev = false;
    if (is_pinned_or_device(src, &dev)) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, E.stream);
    char *st = (char *)E.h_stage + stage_off;
    std::memcpy(st, src, bytes);
    stage_off += (bytes + 255) & ~(size_t)255;
    return cudaMemcpyAsync(dst, st, bytes, cudaMemcpyHostToDevice, E.stream);
}

int estimate_cap(const nnp_batch *b, double rc, int64_t n_ghost)
{
    double pmax = 16.0;
    for (int s = 0; s < b->n_struct; ++s) {
        const int64_t n = b->atom_off[s + 1] - b->atom_off[s];
        if (n <= 0) continue;
        double p;
        if (b->pbc) {
            const double *c = b->cell + 9 * (int64_t)s;
            const double V = std::fabs(c[0] * (c[4] * c[8] - c[5] * c[7]) - c[1] * (c[3] * c[8] - c[5] * c[6]) +
                                       c[2] * (c[3] * c[7] - c[4] * c[6]));
            p = V > 0 ? 4.18879020478639 * rc * rc * rc * (double)n / V : 256.0;
        } else if (n_ghost > 0) {
            // local + ghost atoms: the density of the local atoms' bounding box
            const int64_t a0 = b->atom_off[s], nl = std::max<int64_t>(n - n_ghost, 1);
            double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
            for (int64_t a = a0; a < a0 + nl; ++a)
                for (int d = 0; d < 3; ++d) {
                    lo[d] = std::min(lo[d], b->pos[3 * a + d]);
                    hi[d] = std::max(hi[d], b->pos[3 * a + d]);
                }
            double V = 1.0;
            for (int d = 0; d < 3; ++d) V *= std::max(hi[d] - lo[d], rc);
            p = std::min(4.18879020478639 * rc * rc * rc * (double)nl / V, (double)(n - 1));
        } else {
            p = (double)(n - 1);
        }
        pmax = std::max(pmax, p);
    }
    int cap = (int)std::ceil(1.5 * pmax + 24.0);
    cap = (cap + 7) & ~7;
    return std::min(cap, NNP_MAX_NBR);
}

}  // namespace

extern "C" {

const char *nnp_version(void) { return "nnp_b200 0.1 (sm_100a)"; }

const char *nnp_last_error(const nnp_handle *h) { return h ? h->E.last_error.c_str() : g_create_error.c_str(); }

int nnp_create_from_file(const char *path, nnp_handle **out)
{
    if (!path || !out) return fail(nullptr, NNP_ERR_ARG, "nnp_create_from_file: null argument");
    *out = nullptr;
    std::string text;
    if (!read_file(path, text))
        return fail(nullptr, NNP_ERR_IO, std::string("NNP::read(const char*,NNP&): Could not open nnp file: \"") + path + "\"");
    nnp_handle *h = new nnp_handle();
    std::string msg = nnp::read_potential(text, h->E.host);
    if (!msg.empty()) {
        delete h;
        return fail(nullptr, NNP_ERR_PARSE, msg);
    }
    return finish_create(h, out);
}

int nnp_create_from_basis(int32_t ntypes, const char *const *type_lines, double rc, const char *const *basis_paths,
                          const char *const *network_texts, nnp_handle **out)
{
    if (!out || !type_lines || !basis_paths || !network_texts || ntypes <= 0)
        return fail(nullptr, NNP_ERR_ARG, "nnp_create_from_basis: bad argument");
    if (ntypes > NNP_MAX_TYPES) return fail(nullptr, NNP_ERR_UNSUPPORTED, "too many element types");
    if (!(rc > 0)) return fail(nullptr, NNP_ERR_ARG, "NNP::read(FILE*,NNP&): invalid cutoff.");
    *out = nullptr;
    // a minimal potential text with empty bases, then fill in the pieces
    std::string text = "ann\nntypes " + std::to_string(ntypes) + "\n";
    for (int i = 0; i < ntypes; ++i) text += std::string(type_lines[i]) + "\n";
    nnp_handle *h = new nnp_handle();
    nnp::HostPot &P = h->E.host;
    {
        // parse types with the potential parser by appending an empty rest
        std::istringstream is(text);
        std::string ln;
        std::getline(is, ln);
        std::getline(is, ln);
        P.types.resize(ntypes);
        for (int i = 0; i < ntypes; ++i) {
            std::getline(is, ln);
            std::istringstream ts(ln);
            std::vector<std::string> tok;
            std::string t;
            while (ts >> t) tok.push_back(t);
            P.types[i].name = "NONE";
            for (size_t k = 0; k + 1 < tok.size(); k += 2) {
                std::string tag = tok[k];
                for (auto &c : tag) c = (char)toupper((unsigned char)c);
                const double v = std::atof(tok[k + 1].c_str());
                if (tag == "NAME") P.types[i].name = tok[k + 1];
                else if (tag == "ENERGY") P.types[i].energy = v;
                else if (tag == "MASS") P.types[i].mass = v;
                else if (tag == "CHARGE") P.types[i].charge = v;
                else if (tag == "RADIUS") P.types[i].radius = v;
                else if (tag == "Z") P.types[i].z = v;
                else if (tag == "ALPHA") P.types[i].alpha = v;
                else if (tag == "IE") P.types[i].ie = v;
                else if (tag == "RCOV") P.types[i].rcov = v;
                else if (tag == "RVDW") P.types[i].rvdw = v;
                else if (tag == "AMP") P.types[i].amp = v;
            }
        }
    }
    P.rc = rc;
    P.br.assign(ntypes, std::vector<nnp::HostBasisR>(ntypes));
    P.ba.assign(ntypes, std::vector<nnp::HostBasisA>(ntypes * (ntypes + 1) / 2));
    P.nets.assign(ntypes, nnp::HostNet());
    for (int i = 0; i < ntypes; ++i) {
        std::string btxt;
        if (!read_file(basis_paths[i], btxt)) {
            delete h;
            return fail(nullptr, NNP_ERR_IO, std::string("NNP::read_basis(const char*,NNP&,const char*): Could not open nnp file: \"") + basis_paths[i] + "\"");
        }
        std::string msg = nnp::read_basis_file(btxt, P, i);
        if (msg.empty()) msg = nnp::read_network(network_texts[i], P.nets[i]);
        if (msg.empty() && P.nets[i].nodes.front() != P.n_input(i)) msg = "network input size differs from the basis size";
        if (!msg.empty()) {
            delete h;
            return fail(nullptr, NNP_ERR_PARSE, msg);
        }
    }
    return finish_create(h, out);
}

int nnp_destroy(nnp_handle *h)
{
    if (!h) return NNP_OK;
    h->E.free_all();
    delete h;
    return NNP_OK;
}

int nnp_write(const nnp_handle *h, const char *path)
{
    if (!h || !path) return NNP_ERR_ARG;
    const std::string hp = host_params(const_cast<nnp_handle *>(h)->E);
    if (!hp.empty()) return fail(const_cast<nnp_handle *>(h), NNP_ERR_CUDA, hp);
    std::ofstream f(path, std::ios::out | std::ios::binary);
    if (!f) return fail(const_cast<nnp_handle *>(h), NNP_ERR_IO, std::string("NNP::write(const char*,const NNP&): Could not write to nnh file: \"") + path + "\"");
    f << nnp::write_potential(h->E.host);
    return NNP_OK;
}

int nnp_set_precision(nnp_handle *h, int32_t precision)
{
    if (!h) return NNP_ERR_ARG;
    if (precision != NNP_PREC_FP32 && precision != NNP_PREC_BF16 && precision != NNP_PREC_BF16X3)
        return fail(h, NNP_ERR_ARG, "unknown precision");
    h->E.precision = precision;
    return NNP_OK;
}

int nnp_set_specialization(nnp_handle *h, int32_t enable)
{
    if (!h) return NNP_ERR_ARG;
    nnp::Engine &E = h->E;
    if (enable && !E.jit_module) {
        E.jit_error = nnp::jit_build(E);
        if (!E.jit_error.empty()) {
            E.use_jit = false;
            return fail(h, NNP_ERR_CUDA, E.jit_error);
        }
    }
    E.use_jit = enable != 0;
    return NNP_OK;
}

int nnp_specialization(const nnp_handle *h, int32_t *active, const char **source)
{
    if (!h || !active) return NNP_ERR_ARG;
    *active = (h->E.use_jit && h->E.jit_module) ? 1 : 0;
    if (source) *source = h->E.jit_source.c_str();
    return NNP_OK;
}

int nnp_specialization_check(const char *potential_path, char *log, int32_t log_len)
{
    auto put = [&](const std::string &s) {
        if (log && log_len > 0) {
            std::strncpy(log, s.c_str(), (size_t)log_len - 1);
            log[log_len - 1] = '\0';
        }
    };
    if (!potential_path) return NNP_ERR_ARG;
    std::string text;
    if (!read_file(potential_path, text)) {
        put("could not open potential file");
        return NNP_ERR_IO;
    }
    nnp::Engine E;
    std::string msg = nnp::read_potential(text, E.host);
    if (!msg.empty()) {
        put(msg);
        return NNP_ERR_PARSE;
    }
    msg = E.build_tables();
    if (!msg.empty()) {
        put(msg);
        return NNP_ERR_UNSUPPORTED;
    }
    std::string src;
    std::vector<char> cubin;
    nnp::jit_last_log().clear();
    nnp::tune_from_env(E.tune);
    msg = nnp::jit_compile(E, src, cubin);
    put(msg.empty() ? nnp::jit_last_log() + "\n" + src : msg);
    return msg.empty() ? NNP_OK : NNP_ERR_CUDA;
}

int nnp_set_graphs(nnp_handle *h, int32_t enable)
{
    if (!h) return NNP_ERR_ARG;
    h->E.graph_release();
    h->E.use_graphs = enable != 0;
    return NNP_OK;
}

int nnp_set_accumulation(nnp_handle *h, int32_t acc)
{
    if (!h) return NNP_ERR_ARG;
    if (acc != NNP_ACC_FP32 && acc != NNP_ACC_FP64 && acc != NNP_SYMM_FP64)
        return fail(h, NNP_ERR_ARG, "unknown accumulation mode");
    h->E.acc64 = (acc == NNP_ACC_FP64);
    h->E.symm64 = (acc == NNP_SYMM_FP64);
    return NNP_OK;
}

int nnp_set_stream(nnp_handle *h, void *cuda_stream)
{
    if (!h) return NNP_ERR_ARG;
    nnp::Engine &E = h->E;
    if (E.own_stream && E.stream) cudaStreamDestroy(E.stream);
    E.own_stream = false;
    E.stream = (cudaStream_t)cuda_stream;
    if (!E.stream) {
        cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking);
        E.own_stream = true;
    }
    return NNP_OK;
}

int nnp_ntypes(const nnp_handle *h, int32_t *ntypes)
{
    if (!h || !ntypes) return NNP_ERR_ARG;
    *ntypes = h->E.host.ntypes();
    return NNP_OK;
}

int nnp_type_index(const nnp_handle *h, const char *name, int32_t *index)
{
    if (!h || !name || !index) return NNP_ERR_ARG;
    for (int i = 0; i < h->E.host.ntypes(); ++i)
        if (h->E.host.types[i].name == name) {
            *index = i;
            return NNP_OK;
        }
    *index = -1;
    return fail(const_cast<nnp_handle *>(h), NNP_ERR_TYPE, std::string("unknown element ") + name);
}

int nnp_rc(const nnp_handle *h, double *rc)
{
    if (!h || !rc) return NNP_ERR_ARG;
    *rc = h->E.host.rc;
    return NNP_OK;
}

int nnp_n_input(const nnp_handle *h, int32_t type, int32_t *n_input)
{
    if (!h || !n_input || type < 0 || type >= h->E.host.ntypes()) return NNP_ERR_ARG;
    *n_input = h->E.host.n_input(type);
    return NNP_OK;
}

int nnp_nparams(const nnp_handle *h, int32_t type, int32_t *n)
{
    if (!h || !n) return NNP_ERR_ARG;
    if (type < 0) {
        int s = 0;
        for (const auto &net : h->E.host.nets) s += net.nparams();
        *n = s;
        return NNP_OK;
    }
    if (type >= h->E.host.ntypes()) return NNP_ERR_ARG;
    *n = h->E.host.nets[type].nparams();
    return NNP_OK;
}

int nnp_get_params(const nnp_handle *h, double *params)
{
    if (!h || !params) return NNP_ERR_ARG;
    const std::string hp = host_params(const_cast<nnp_handle *>(h)->E);
    if (!hp.empty()) return fail(const_cast<nnp_handle *>(h), NNP_ERR_CUDA, hp);
    size_t k = 0;
    for (const auto &net : h->E.host.nets) {
        const int nl = (int)net.nodes.size() - 1;
        for (int l = 0; l < nl; ++l)
            for (double v : net.b[l]) params[k++] = v;
        for (int l = 0; l < nl; ++l) {
            const int ni = net.nodes[l], no = net.nodes[l + 1];
            for (int m = 0; m < ni; ++m)
                for (int n = 0; n < no; ++n) params[k++] = net.w[l][(size_t)n * ni + m];
        }
    }
    return NNP_OK;
}

int nnp_set_params(nnp_handle *h, const double *params)
{
    if (!h || !params) return NNP_ERR_ARG;
    h->E.host_stale = false;          // every parameter is overwritten here
    size_t k = 0;
    for (auto &net : h->E.host.nets) {
        const int nl = (int)net.nodes.size() - 1;
        for (int l = 0; l < nl; ++l)
            for (auto &v : net.b[l]) v = params[k++];
        for (int l = 0; l < nl; ++l) {
            const int ni = net.nodes[l], no = net.nodes[l + 1];
            for (int m = 0; m < ni; ++m)
                for (int n = 0; n < no; ++n) net.w[l][(size_t)n * ni + m] = params[k++];
        }
    }
    std::string msg = h->E.upload();
    if (!msg.empty()) return fail(h, NNP_ERR_CUDA, msg);
    return NNP_OK;
}

}  // extern "C"

namespace {

// nnp_compute and nnp_compute_md: the whole pipeline, with the optional
// per-atom energies [N] and per-structure virials [9 S] of the MD call.
// internal flag of compute_impl: energies and forces are computed into the
// handle's buffers (e_struct, force) and the output pointers may be NULL
constexpr uint32_t KEEP_ON_DEVICE = 1u << 30;

int compute_impl(nnp_handle *h, const nnp_batch *b, double *energy, double *forces, double *symm_out,
                 double *atom_energy, double *virial, uint32_t flags, int64_t n_ghost = 0)
{
    if (!h || !b) return NNP_ERR_ARG;
    nnp::Engine &E = h->E;
    E.n_ghost = n_ghost;
    if (b->n_struct < 0) return fail(h, NNP_ERR_ARG, "negative structure count");
    if ((flags & NNP_ENERGY) && !energy && !(flags & KEEP_ON_DEVICE)) return fail(h, NNP_ERR_ARG, "energy output missing");
    if ((flags & NNP_FORCES) && !forces && !(flags & KEEP_ON_DEVICE)) return fail(h, NNP_ERR_ARG, "force output missing");
    if ((flags & NNP_SYMM) && !symm_out) return fail(h, NNP_ERR_ARG, "symmetry-function output missing");
    const int S = b->n_struct;
    if (S == 0) return NNP_OK;
    if (!b->atom_off || !b->pos || !b->type || (b->pbc && !b->cell)) return fail(h, NNP_ERR_ARG, "batch array missing");
    const bool devp = (flags & NNP_DEVICE_PTRS) != 0;
    int64_t N = 0;
    cudaError_t ce = cudaSuccess;
    auto chk = [&](cudaError_t x) { if (x != cudaSuccess && ce == cudaSuccess) ce = x; };
    if (!devp) {
        if (b->atom_off[0] != 0) return fail(h, NNP_ERR_ARG, "atom_off[0] must be 0");
        for (int s = 0; s < S; ++s)
            if (b->atom_off[s + 1] < b->atom_off[s]) return fail(h, NNP_ERR_ARG, "atom_off must be non-decreasing");
        N = b->atom_off[S];
        if (N >= (int64_t)1 << 28) return fail(h, NNP_ERR_CAPACITY, "more than 2^28 atoms in one batch");
        const int T = E.host.ntypes();
        // a branch-free pass (vectorised), then the first bad atom for the message
        unsigned any_bad = 0;
        for (int64_t i = 0; i < N; ++i) any_bad |= (unsigned)b->type[i] >= (unsigned)T;
        if (any_bad)
            for (int64_t i = 0; i < N; ++i)
                if (b->type[i] < 0 || b->type[i] >= T)
                    return fail(h, NNP_ERR_TYPE, "atom " + std::to_string(i) + " has type index " + std::to_string(b->type[i]) + " outside [0," + std::to_string(T) + ")");
        E.cap = std::max(E.cap, estimate_cap(b, E.host.rc, n_ghost));
        // inputs -> device
        const size_t bo = sizeof(int64_t) * (S + 1), bp = sizeof(double) * 3 * N, bt = sizeof(int32_t) * N,
                     bc = b->pbc ? sizeof(double) * 9 * S : 0;
        if (stage_bytes(E, bo + bp + bt + bc + 4 * 256) != NNP_OK) return fail(h, NNP_ERR_CUDA, "cudaMallocHost failed");
        chk(E.atom_off.reserve(S + 1));
        chk(E.pos.reserve(3 * std::max<int64_t>(N, 1)));
        chk(E.type.reserve(std::max<int64_t>(N, 1)));
        chk(E.cell.reserve(9 * (size_t)S));
        if (ce != cudaSuccess) return fail(h, NNP_ERR_CUDA, std::string("device allocation failed: ") + cudaGetErrorString(ce));
        size_t so = 0;
        chk(h2d(E, E.atom_off.p, b->atom_off, bo, so));
        chk(h2d(E, E.pos.p, b->pos, bp, so));
        chk(h2d(E, E.type.p, b->type, bt, so));
        if (b->pbc) chk(h2d(E, E.cell.p, b->cell, bc, so));
        if (ce != cudaSuccess) return fail(h, NNP_ERR_CUDA, std::string("input copy failed: ") + cudaGetErrorString(ce));
    } else {
        int64_t n = 0;
        chk(cudaMemcpyAsync(&n, b->atom_off + S, sizeof n, cudaMemcpyDeviceToHost, E.stream));
        chk(cudaStreamSynchronize(E.stream));
        if (ce != cudaSuccess) return fail(h, NNP_ERR_CUDA, std::string("reading atom count failed: ") + cudaGetErrorString(ce));
        N = n;
        if (N < 0 || N >= (int64_t)1 << 28) return fail(h, NNP_ERR_ARG, "bad atom count in atom_off");
        if (E.cap < 128) E.cap = 128;
        // run on the caller's arrays in place
    }
    // kernels read through these
    nnp::DBuf<int64_t> u_off = E.atom_off;
    nnp::DBuf<double> u_pos = E.pos, u_cell = E.cell;
    nnp::DBuf<int> u_type = E.type;
    if (devp) {
        E.atom_off.p = const_cast<int64_t *>(b->atom_off);
        E.pos.p = const_cast<double *>(b->pos);
        E.type.p = const_cast<int32_t *>(b->type);
        E.cell.p = const_cast<double *>(b->cell);
    }
    E.want_virial = (virial != nullptr);
    if (virial) chk(E.vir.reserve(9 * (size_t)S));
    if (atom_energy && !devp) chk(E.eatom_d.reserve(std::max<int64_t>(N, 1)));
    if (ce != cudaSuccess) {
        E.want_virial = false;
        return fail(h, NNP_ERR_CUDA, std::string("device allocation failed: ") + cudaGetErrorString(ce));
    }
    int rc = NNP_OK;
    // the device-side step: every launch depends only on host-known sizes and
    // the handle's buffers, so it can be captured as one CUDA graph
    auto step = [&]() -> std::string {
        std::string msg = nnp::run_prepare(E, N, S, b->pbc);
        if (msg.empty()) msg = nnp::run_neighbors(E, b->pbc);
        if (msg.empty()) msg = nnp::run_symm(E);
        if (msg.empty() && ((flags & (NNP_ENERGY | NNP_FORCES)) || atom_energy || virial)) msg = nnp::run_nn(E);
        if (msg.empty() && ((flags & NNP_FORCES) || virial)) msg = nnp::run_force(E);
        if (msg.empty() && (flags & NNP_ENERGY)) msg = nnp::run_energy(E, (flags & NNP_VACUUM) != 0);
        return msg;
    };
    // Graph replay: after a call has run eagerly (so every buffer has its
    // size), the next call with the same key is captured once and then
    // replayed.  Not on the legacy default stream (it cannot be captured),
    // and not while the stage timers are on.
    bool graphs = E.use_graphs && !E.timing && E.stream != nullptr && E.stream != cudaStreamLegacy &&
                  E.stream != cudaStreamPerThread;
    std::vector<int64_t> key;
    if (graphs)
        key = {N, S, b->pbc, n_ghost, E.cap, (int64_t)flags, (int64_t)(atom_energy != nullptr), (int64_t)(virial != nullptr),
               E.precision, (int64_t)(intptr_t)(E.use_jit ? E.jit_symm : nullptr), (int64_t)E.acc64 + 2 * E.symm64,
               (int64_t)(intptr_t)E.atom_off.p,
               (int64_t)(intptr_t)E.pos.p, (int64_t)(intptr_t)E.type.p, (int64_t)(intptr_t)E.cell.p,
               (int64_t)(intptr_t)E.nbr.p, (int64_t)(intptr_t)E.G.p, (int64_t)(intptr_t)E.force.p,
               (int64_t)(intptr_t)E.e_struct.p, (int64_t)(intptr_t)E.e_atom.p, (int64_t)(intptr_t)E.vir.p};
    for (int attempt = 0; attempt < 4; ++attempt) {
        std::string msg;
        if (graphs && E.graph_exec && key == E.graph_key) {
            chk(cudaGraphLaunch((cudaGraphExec_t)E.graph_exec, E.stream));
            E.launches += E.graph_launches;
        } else if (graphs && key == E.graph_key) {
            // second call with this key: capture, then replay
            const int64_t l0 = E.launches;
            cudaGraph_t graph = nullptr;
            cudaError_t g = cudaStreamBeginCapture(E.stream, cudaStreamCaptureModeThreadLocal);
            if (g == cudaSuccess) {
                msg = step();
                g = cudaStreamEndCapture(E.stream, &graph);
            }
            cudaGraphExec_t exec = nullptr;
            if (g == cudaSuccess && msg.empty()) g = cudaGraphInstantiate(&exec, graph, 0);
            if (graph) cudaGraphDestroy(graph);
            if (g == cudaSuccess && msg.empty() && exec) {
                E.graph_exec = exec;
                E.graph_launches = E.launches - l0;
                E.launches = l0;
                chk(cudaGraphLaunch(exec, E.stream));
                E.launches += E.graph_launches;
            } else {
                // capture not possible here: run eagerly from now on
                cudaGetLastError();
                if (exec) cudaGraphExecDestroy(exec);
                E.use_graphs = false;
                E.launches = l0;
                msg = step();
            }
        } else {
            if (graphs) {
                E.graph_release();
                E.graph_key = key;        // capture on the next call with this key
            }
            msg = step();
        }
        if (!msg.empty()) { rc = fail(h, NNP_ERR_CUDA, msg); break; }
        chk(cudaMemcpyAsync(E.h_err, E.err.p, sizeof(nnp::DevErr), cudaMemcpyDeviceToHost, E.stream));
        chk(cudaStreamSynchronize(E.stream));
        if (ce != cudaSuccess) { rc = fail(h, NNP_ERR_CUDA, std::string("kernel failure: ") + cudaGetErrorString(ce)); break; }
        const nnp::DevErr er = *E.h_err;
        if (er.bad_type) { rc = fail(h, NNP_ERR_TYPE, "atom type index out of range"); break; }
        if (er.bad_cell == 1) { rc = fail(h, NNP_ERR_ARG, "a periodic cell has zero volume"); break; }
        if (er.bad_cell) {
            rc = fail(h, NNP_ERR_CAPACITY, "a periodic cell is thinner than rc/" + std::to_string(NNP_MAX_IMAGES) +
                                               " in some direction (too many images to search)");
            break;
        }
        if (er.need_cap > E.cap) {
            if (er.need_cap > NNP_MAX_NBR) {
                rc = fail(h, NNP_ERR_CAPACITY, "an atom has " + std::to_string(er.need_cap) + " neighbours; the device path handles up to " + std::to_string(NNP_MAX_NBR));
                break;
            }
            E.cap = std::min(NNP_MAX_NBR, ((er.need_cap + er.need_cap / 8 + 8) + 7) & ~7);
            // the graph was made for the old capacity: drop it, retry eagerly
            E.graph_release();
            graphs = false;
            continue;
        }
        if (er.nonfinite == 2) { rc = fail(h, NNP_ERR_CUDA, "tensor-core network kernel: an MMA wait timed out"); break; }
        if (er.nonfinite) { rc = fail(h, NNP_ERR_NOT_FINITE, "non-finite energy or force"); }
        // autotuning on and this capacity class not tuned yet: time the
        // candidate kernels on this batch, then run the step again with the
        // chosen ones (the class is marked tuned, so this happens once)
        if (rc == NNP_OK && E.autotune && E.use_jit && E.jit_module && (flags & NNP_FORCES) &&
            nnp::tune_needed(E, E.cap)) {
            const std::string tm = nnp::autotune(E, E.cap, step);
            E.graph_release();
            graphs = false;
            if (!tm.empty()) { rc = fail(h, NNP_ERR_CUDA, tm); break; }
            continue;
        }
        // outputs
        if (!devp) {
            const size_t be = sizeof(double) * S, bf = sizeof(double) * 3 * N;
            if ((flags & NNP_ENERGY) && energy) chk(cudaMemcpyAsync(energy, E.e_struct.p, be, cudaMemcpyDeviceToHost, E.stream));
            if ((flags & NNP_FORCES) && forces) chk(cudaMemcpyAsync(forces, E.force.p, bf, cudaMemcpyDeviceToHost, E.stream));
            if (flags & NNP_SYMM) {
                chk(E.symm_d.reserve((size_t)N * E.gstride + 1));
                nnp::run_symm_to_double(E, E.symm_d.p);
                chk(cudaMemcpyAsync(symm_out, E.symm_d.p, sizeof(double) * N * E.gstride, cudaMemcpyDeviceToHost, E.stream));
            }
            if (atom_energy) {
                nnp::run_atom_energy(E, (flags & NNP_VACUUM) != 0, E.eatom_d.p);
                chk(cudaMemcpyAsync(atom_energy, E.eatom_d.p, sizeof(double) * (N - n_ghost), cudaMemcpyDeviceToHost,
                                    E.stream));
            }
            if (virial) chk(cudaMemcpyAsync(virial, E.vir.p, sizeof(double) * 9 * S, cudaMemcpyDeviceToHost, E.stream));
        } else {
            if ((flags & NNP_ENERGY) && energy) chk(cudaMemcpyAsync(energy, E.e_struct.p, sizeof(double) * S, cudaMemcpyDeviceToDevice, E.stream));
            if ((flags & NNP_FORCES) && forces) chk(cudaMemcpyAsync(forces, E.force.p, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, E.stream));
            if (flags & NNP_SYMM) nnp::run_symm_to_double(E, symm_out);
            if (atom_energy) nnp::run_atom_energy(E, (flags & NNP_VACUUM) != 0, atom_energy);
            if (virial) chk(cudaMemcpyAsync(virial, E.vir.p, sizeof(double) * 9 * S, cudaMemcpyDeviceToDevice, E.stream));
        }
        chk(cudaStreamSynchronize(E.stream));
        if (ce != cudaSuccess) rc = fail(h, NNP_ERR_CUDA, std::string("output copy failed: ") + cudaGetErrorString(ce));
        break;
    }
    if (devp) {
        E.atom_off = u_off;
        E.pos = u_pos;
        E.cell = u_cell;
        E.type = u_type;
    }
    E.want_virial = false;
    return rc;
}

}  // namespace

extern "C" {

int nnp_compute(nnp_handle *h, const nnp_batch *b, double *energy, double *forces, double *symm_out, uint32_t flags)
{
    return compute_impl(h, b, energy, forces, symm_out, nullptr, nullptr, flags);
}

int nnp_compute_md(nnp_handle *h, const nnp_batch *b, double *energy, double *forces, double *atom_energy,
                   double *virial, uint32_t flags)
{
    if (!h || !b) return NNP_ERR_ARG;
    if (flags & ~(uint32_t)(NNP_VACUUM | NNP_DEVICE_PTRS)) return fail(h, NNP_ERR_ARG, "flags other than NNP_VACUUM and NNP_DEVICE_PTRS");
    if (!energy && !forces && !atom_energy && !virial) return fail(h, NNP_ERR_ARG, "no output requested");
    flags |= (energy ? NNP_ENERGY : 0u) | (forces ? NNP_FORCES : 0u);
    return compute_impl(h, b, energy, forces, nullptr, atom_energy, virial, flags);
}

int nnp_type_name(const nnp_handle *h, int32_t type, const char **name)
{
    if (!h || !name || type < 0 || type >= h->E.host.ntypes()) return NNP_ERR_ARG;
    *name = h->E.host.types[type].name.c_str();
    return NNP_OK;
}

int nnp_read_structures(int32_t ntypes, const char *const *type_names, const char *path, int32_t format,
                        int32_t *n_struct, int64_t *n_atoms, int64_t *atom_off, double *pos, int32_t *type,
                        double *cell, int32_t *pbc, double *energy, double *forces)
{
    auto bad = [](int code, const std::string &m) {
        g_create_error = m;
        return code;
    };
    if (ntypes < 0 || (ntypes > 0 && !type_names) || !path || !n_struct || !n_atoms) return bad(NNP_ERR_ARG, "bad argument");
    if (format != NNP_FMT_XYZ && format != NNP_FMT_VASP) return bad(NNP_ERR_ARG, "unknown structure format");
    std::string text;
    if (!read_file(path, text)) return bad(NNP_ERR_IO, std::string("Could not open file: ") + path);
    std::vector<nnp::ReadStruct> rs;
    const std::string msg = format == NNP_FMT_XYZ ? nnp::read_xyz_frames(text, rs) : nnp::read_vasp(text, rs);
    if (!msg.empty()) return bad(NNP_ERR_PARSE, msg);
    int64_t N = 0;
    for (const auto &r : rs) N += (int64_t)r.names.size();
    if (atom_off) {
        if (*n_struct < (int32_t)rs.size() || *n_atoms < N)
            return bad(NNP_ERR_CAPACITY, "output arrays hold fewer structures or atoms than the file");
        int64_t a = 0;
        atom_off[0] = 0;
        for (size_t s = 0; s < rs.size(); ++s) {
            const nnp::ReadStruct &r = rs[s];
            for (size_t i = 0; i < r.names.size(); ++i, ++a) {
                int t = -1;
                for (int k = 0; k < ntypes; ++k)
                    if (type_names[k] && r.names[i] == type_names[k]) t = k;
                if (t < 0) return bad(NNP_ERR_TYPE, "element \"" + r.names[i] + "\" is not in the potential");
                if (type) type[a] = t;
                if (pos)
                    for (int d = 0; d < 3; ++d) pos[3 * a + d] = r.pos[3 * i + d];
                if (forces)
                    for (int d = 0; d < 3; ++d) forces[3 * a + d] = r.forces[3 * i + d];
            }
            atom_off[s + 1] = a;
            if (cell)
                for (int k = 0; k < 9; ++k) cell[9 * s + k] = r.cell[k];
            if (pbc) pbc[s] = r.pbc ? 1 : 0;
            if (energy) energy[s] = r.energy;
        }
    }
    *n_struct = (int32_t)rs.size();
    *n_atoms = N;
    return NNP_OK;
}

int nnp_input_stats(nnp_handle *h, const nnp_batch *batch, int64_t *count, double *stats)
{
    if (!h || !batch || !count || !stats) return NNP_ERR_ARG;
    nnp::Engine &E = h->E;
    if (batch->n_struct <= 0) return fail(h, NNP_ERR_ARG, "empty batch");
    // neighbour lists and symmetry functions of the batch (no networks)
    int rc = compute_impl(h, batch, nullptr, nullptr, nullptr, nullptr, nullptr, 0u);
    if (rc != NNP_OK) return rc;
    std::vector<int64_t> c;
    std::vector<double> st;
    const std::string msg = nnp::run_input_stats(E, c, st);
    if (!msg.empty()) return fail(h, NNP_ERR_CUDA, msg);
    std::copy(c.begin(), c.end(), count);
    std::copy(st.begin(), st.end(), stats);
    return NNP_OK;
}

int nnp_precondition(nnp_handle *h, const nnp_batch *batch, int32_t prebias, int32_t prescale, double inbias,
                     double inscale)
{
    if (!h || !batch) return NNP_ERR_ARG;
    if (prebias < NNP_PREBIAS_IDENTITY || prebias > NNP_PREBIAS_MIN) return fail(h, NNP_ERR_ARG, "Invalid input bias.");
    if (prescale < NNP_PRESCALE_IDENTITY || prescale > NNP_PRESCALE_MAX)
        return fail(h, NNP_ERR_ARG, "Invalid input scaling.");
    nnp::Engine &E = h->E;
    const std::string hp = host_params(E);
    if (!hp.empty()) return fail(h, NNP_ERR_CUDA, hp);
    const int T = E.host.ntypes(), gs = E.gstride;
    std::vector<int64_t> cnt(T);
    std::vector<double> st((size_t)T * NNP_NSTATS * gs);
    int rc = nnp_input_stats(h, batch, cnt.data(), st.data());
    if (rc != NNP_OK) return rc;
    auto S = [&](int t, int s, int k) { return st[((size_t)t * NNP_NSTATS + s) * gs + k]; };
    for (int t = 0; t < T; ++t) {
        nnp::HostNet &net = E.host.nets[t];
        const int nin = (int)net.inpb.size();
        for (int k = 0; k < nin; ++k) {
            double b = 0.0;
            switch (prebias) {
            case NNP_PREBIAS_MEAN: b = -S(t, NNP_STAT_MEAN, k); break;
            case NNP_PREBIAS_HAR: b = -S(t, NNP_STAT_HARMONIC, k); break;
            case NNP_PREBIAS_RMS: b = -S(t, NNP_STAT_RMS, k); break;
            case NNP_PREBIAS_MID: b = -0.5 * (S(t, NNP_STAT_MAX, k) + S(t, NNP_STAT_MIN, k)); break;
            case NNP_PREBIAS_MIN: b = -S(t, NNP_STAT_MIN, k); break;
            default: b = 0.0; break;
            }
            double w = 1.0;
            switch (prescale) {
            case NNP_PRESCALE_DEV: {
                const double d = S(t, NNP_STAT_DEV, k);
                w = (d == 0) ? 1.0 : 1.0 / d;
            } break;
            case NNP_PRESCALE_MINMAX: {
                const double d = S(t, NNP_STAT_MAX, k) - S(t, NNP_STAT_MIN, k);
                w = (d > 0) ? 1.0 / d : 1.0;
            } break;
            case NNP_PRESCALE_MAX: {
                const double d = S(t, NNP_STAT_MAX, k);
                w = (d > 0) ? 1.0 / d : 1.0;
            } break;
            default: w = 1.0; break;
            }
            net.inpb[k] = b + inbias;
            net.inpw[k] = w * inscale;
        }
        for (auto &v : net.outb) v = 0.0;
        for (auto &v : net.outw) v = 1.0;
    }
    const std::string msg = E.upload();
    if (!msg.empty()) return fail(h, NNP_ERR_CUDA, msg);
    return NNP_OK;
}

int nnp_taylor_expand(int32_t n_struct, const int64_t *atom_off, const double *pos, const int32_t *type,
                      const double *energy, const double *forces, int32_t nadd, int32_t dist, double rdelta,
                      uint64_t seed, int64_t *out_atom_off, double *out_pos, int32_t *out_type, double *out_energy,
                      int32_t *out_src, int32_t *n_out)
{
    auto bad = [](int code, const std::string &m) {
        g_create_error = m;
        return code;
    };
    if (n_struct < 0 || nadd < 0 || !n_out) return bad(NNP_ERR_ARG, "bad structure count, copy count or output");
    if (n_struct > 0 && (!atom_off || !pos || !type || !energy || !forces))
        return bad(NNP_ERR_ARG, "input array missing");
    if (!out_atom_off || !out_pos || !out_type || !out_energy || !out_src) return bad(NNP_ERR_ARG, "output array missing");
    if (!(dist == 1 || dist == 2 || dist == 3 || dist == 5 || dist == 6 || dist == 7))
        return bad(NNP_ERR_ARG, "Invalid position distribution.");
    if (!(rdelta >= 0.0) || !std::isfinite(rdelta)) return bad(NNP_ERR_ARG, "rdelta must be finite and non-negative");
    if (n_struct == 0) {
        out_atom_off[0] = 0;
        *n_out = 0;
        return NNP_OK;
    }
    if (atom_off[0] != 0) return bad(NNP_ERR_ARG, "atom_off[0] must be 0");
    for (int s = 0; s < n_struct; ++s)
        if (atom_off[s + 1] < atom_off[s]) return bad(NNP_ERR_ARG, "atom_off must be non-decreasing");
    std::vector<int64_t> oo;
    std::vector<int> src;
    std::vector<double> op, oe;
    const std::string msg = nnp::taylor_expand(n_struct, atom_off, pos, energy, forces, nadd, dist, rdelta, seed, oo,
                                               src, op, oe);
    if (!msg.empty()) return bad(NNP_ERR_CUDA, msg);
    const int O = (int)src.size();
    std::copy(oo.begin(), oo.end(), out_atom_off);
    std::copy(op.begin(), op.end(), out_pos);
    std::copy(oe.begin(), oe.end(), out_energy);
    for (int o = 0; o < O; ++o) {
        out_src[o] = src[o];
        const int64_t a0 = atom_off[src[o]], n = atom_off[src[o] + 1] - a0;
        std::copy(type + a0, type + a0 + n, out_type + oo[o]);
    }
    *n_out = O;
    return NNP_OK;
}

int nnp_compute_local_ghost(nnp_handle *h, int64_t n_local, int64_t n_ghost, const double *pos,
                            const int32_t *type, double *energy, double *forces, double *atom_energy, double *virial,
                            uint32_t flags)
{
    if (!h) return NNP_ERR_ARG;
    if (flags & ~(uint32_t)NNP_VACUUM) return fail(h, NNP_ERR_ARG, "flags other than NNP_VACUUM");
    if (n_local < 0 || n_ghost < 0) return fail(h, NNP_ERR_ARG, "negative atom count");
    if (!energy && !forces && !atom_energy && !virial) return fail(h, NNP_ERR_ARG, "no output requested");
    if (n_local + n_ghost == 0) {
        if (energy) *energy = 0.0;
        if (virial)
            for (int k = 0; k < 9; ++k) virial[k] = 0.0;
        return NNP_OK;
    }
    if (!pos || !type) return fail(h, NNP_ERR_ARG, "positions and types are required");
    const int64_t off[2] = {0, n_local + n_ghost};
    const nnp_batch b = {1, off, pos, type, nullptr, 0};
    flags |= (energy ? NNP_ENERGY : 0u) | (forces ? NNP_FORCES : 0u);
    return compute_impl(h, &b, energy, forces, nullptr, atom_energy, virial, flags, n_ghost);
}

int nnp_energy_symm_noalloc(nnp_handle *h, int32_t n_struct, int64_t n_atoms, const int64_t *d_atom_off,
                            const int32_t *d_type, const float *d_symm, int32_t gstride, uint32_t flags,
                            double *d_energy)
{
    if (!h) return NNP_ERR_ARG;
    nnp::Engine &E = h->E;
    if (n_struct < 0 || n_atoms < 0) return fail(h, NNP_ERR_ARG, "negative structure or atom count");
    if (flags & ~(uint32_t)NNP_VACUUM) return fail(h, NNP_ERR_ARG, "flags other than NNP_VACUUM");
    if (n_atoms > NNP_NOALLOC_MAX_ATOMS)
        return fail(h, NNP_ERR_CAPACITY, "allocation-free call takes at most " + std::to_string(NNP_NOALLOC_MAX_ATOMS) +
                                             " atoms, got " + std::to_string(n_atoms));
    if (E.precision != NNP_PREC_FP32) return fail(h, NNP_ERR_UNSUPPORTED, "the allocation-free call runs the FP32 networks only (set precision to FP32)");
    int nin = 0;
    for (int t = 0; t < E.dpot.ntypes; ++t) nin = std::max(nin, E.dpot.t[t].n_input);
    if (gstride < nin) return fail(h, NNP_ERR_ARG, "gstride " + std::to_string(gstride) + " is below the largest input size " + std::to_string(nin));
    if (n_struct == 0) return NNP_OK;
    if (!d_atom_off || !d_energy || (n_atoms > 0 && (!d_type || !d_symm))) return fail(h, NNP_ERR_ARG, "null device pointer");
    // the handle's tables live on the device it was created on; that device must be current
    cudaPointerAttributes pa;
    int dev = -1;
    if (cudaPointerGetAttributes(&pa, E.d_pot) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess || pa.device != dev) {
        cudaGetLastError();
        return fail(h, NNP_ERR_ARG, "the handle's device is not the current device");
    }
    std::string msg = nnp::run_energy_symm_noalloc(E, n_struct, n_atoms, d_atom_off, d_type, d_symm, gstride,
                                                   (flags & NNP_VACUUM) != 0, d_energy);
    return msg.empty() ? NNP_OK : fail(h, NNP_ERR_CUDA, msg);
}

int nnp_compute_energy_symm(nnp_handle *h, int32_t n_struct, const int64_t *atom_off, const int32_t *type,
                            const double *symm, int32_t gstride, double *energy)
{
    if (!h || !atom_off || !type || !symm || !energy || n_struct < 0) return NNP_ERR_ARG;
    nnp::Engine &E = h->E;
    if (n_struct == 0) return NNP_OK;
    const int64_t N = atom_off[n_struct];
    const int T = E.host.ntypes();
    for (int64_t i = 0; i < N; ++i)
        if (type[i] < 0 || type[i] >= T) return fail(h, NNP_ERR_TYPE, "atom type index out of range");
    if (gstride < E.gstride) {
        // repack to the device row length
    }
    cudaError_t ce = cudaSuccess;
    auto chk = [&](cudaError_t x) { if (x != cudaSuccess && ce == cudaSuccess) ce = x; };
    std::string msg = nnp::run_prepare(E, N, n_struct, 0);
    if (!msg.empty()) return fail(h, NNP_ERR_CUDA, msg);
    chk(E.atom_off.reserve(n_struct + 1));
    chk(E.type.reserve(std::max<int64_t>(N, 1)));
    chk(E.symm_d.reserve((size_t)std::max<int64_t>(N, 1) * E.gstride));
    if (ce != cudaSuccess) return fail(h, NNP_ERR_CUDA, "device allocation failed");
    std::vector<double> rows((size_t)N * E.gstride, 0.0);
    for (int64_t i = 0; i < N; ++i)
        for (int g = 0; g < std::min<int>(gstride, E.gstride); ++g) rows[(size_t)i * E.gstride + g] = symm[(size_t)i * gstride + g];
    chk(cudaMemcpyAsync(E.atom_off.p, atom_off, sizeof(int64_t) * (n_struct + 1), cudaMemcpyHostToDevice, E.stream));
    chk(cudaMemcpyAsync(E.type.p, type, sizeof(int32_t) * N, cudaMemcpyHostToDevice, E.stream));
    chk(cudaMemcpyAsync(E.symm_d.p, rows.data(), sizeof(double) * rows.size(), cudaMemcpyHostToDevice, E.stream));
    msg = nnp::run_nn_from_symm(E, E.symm_d.p, E.gstride);
    if (msg.empty()) msg = nnp::run_energy(E, true);
    if (!msg.empty()) return fail(h, NNP_ERR_CUDA, msg);
    chk(cudaMemcpyAsync(energy, E.e_struct.p, sizeof(double) * n_struct, cudaMemcpyDeviceToHost, E.stream));
    chk(cudaStreamSynchronize(E.stream));
    if (ce != cudaSuccess) return fail(h, NNP_ERR_CUDA, std::string("compute_energy failed: ") + cudaGetErrorString(ce));
    return NNP_OK;
}

int nnp_set_timing(nnp_handle *h, int32_t enable)
{
    if (!h) return NNP_ERR_ARG;
    nnp::Engine &E = h->E;
    if (enable && !E.ev[0])
        for (auto &e : E.ev)
            if (cudaEventCreate(&e) != cudaSuccess) return fail(h, NNP_ERR_CUDA, "cudaEventCreate failed");
    E.timing = enable != 0;
    return NNP_OK;
}

int nnp_stage_times(const nnp_handle *h, float *ms, int32_t n)
{
    if (!h || !ms || n < 0) return NNP_ERR_ARG;
    const nnp::Engine &E = h->E;
    for (int k = 0; k < n; ++k) ms[k] = 0.f;
    if (!E.timing) return NNP_OK;
    for (int k = 0; k < n && k < 5; ++k) {
        float t = 0.f;
        if (cudaEventElapsedTime(&t, E.ev[k], E.ev[k + 1]) != cudaSuccess) {
            cudaGetLastError();
            t = 0.f;
        }
        ms[k] = t;
    }
    return NNP_OK;
}

int nnp_neighbor_counts(nnp_handle *h, int32_t *counts)
{
    if (!h || !counts) return NNP_ERR_ARG;
    nnp::Engine &E = h->E;
    const size_t n = (size_t)E.n_atoms * E.dpot.ntypes;
    if (n == 0) return NNP_OK;
    int *d = nullptr;
    if (cudaMalloc((void **)&d, n * sizeof(int)) != cudaSuccess) return fail(h, NNP_ERR_CUDA, "cudaMalloc failed");
    std::string msg = nnp::run_neighbor_counts(E, d);
    cudaError_t ce = cudaMemcpyAsync(counts, d, n * sizeof(int), cudaMemcpyDeviceToHost, E.stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(E.stream);
    cudaFree(d);
    if (!msg.empty()) return fail(h, NNP_ERR_CUDA, msg);
    if (ce != cudaSuccess) return fail(h, NNP_ERR_CUDA, cudaGetErrorString(ce));
    return NNP_OK;
}

int nnp_launch_count(const nnp_handle *h, int64_t *n)
{
    if (!h || !n) return NNP_ERR_ARG;
    *n = h->E.launches;
    return NNP_OK;
}



int nnp_opt_adam(nnp_handle *h, double gamma, double eps)
{
    return opt_adam_impl(h, gamma, eps, -1, 0.0);
}

int nnp_decay_step(int32_t kind, double alpha, int32_t period, double gamma, int32_t step, double *out)
{
    if (!out) return NNP_ERR_ARG;
    switch (kind) {
    case NNP_DECAY_CONST: *out = gamma; break;
    case NNP_DECAY_EXP: *out = gamma * (1.0 - alpha); break;
    case NNP_DECAY_GAUSS: *out = gamma * (1.0 - 2.0 * alpha * step); break;
    case NNP_DECAY_SQRT: *out = gamma * (1.0 - 0.5 * alpha / (1.0 + alpha * step)); break;
    case NNP_DECAY_INV: *out = gamma * (1.0 - alpha / (1.0 + alpha * step)); break;
    case NNP_DECAY_STEP:
        if (period <= 0) {
            g_create_error = "opt::Decay: STEP needs a positive period";
            return NNP_ERR_ARG;
        }
        *out = (step > 0 && (unsigned)step % (unsigned)period == 0) ? gamma * alpha : gamma;
        break;
    default:
        g_create_error = "opt::Decay::step(const Objective&,const Iterator&): invalid decay method.";
        return NNP_ERR_ARG;
    }
    return NNP_OK;
}

int nnp_opt_step(nnp_handle *h, double *gamma, int32_t step, int32_t decay_kind, double alpha, int32_t period,
                 int32_t reg_kind, double eta, double eps)
{
    if (!h || !gamma) return NNP_ERR_ARG;
    if (reg_kind < NNP_REG_LASSO || reg_kind > NNP_REG_NONE) return fail(h, NNP_ERR_ARG, "invalid regularization");
    if (alpha < 0) return fail(h, NNP_ERR_ARG, "opt::Decay::read(Token&): invalid alpha.");
    double g = 0.0;
    if (nnp_decay_step(decay_kind, alpha, period, *gamma, step, &g) != NNP_OK) return fail(h, NNP_ERR_ARG, g_create_error);
    const int rc = opt_adam_impl(h, g, eps, reg_kind == NNP_REG_NONE ? -1 : reg_kind, eta);
    if (rc == NNP_OK) *gamma = g;
    return rc;
}

}  // extern "C"

namespace {
int opt_adam_impl(nnp_handle *h, double gamma, double eps, int reg, double eta)
{
    if (!h) return NNP_ERR_ARG;
    nnp::Engine &E = h->E;
    if (!E.grad_valid) return fail(h, NNP_ERR_ARG, "no gradient: call nnp_train_grad first");
    if (!(gamma >= 0.0) || !std::isfinite(gamma)) return fail(h, NNP_ERR_ARG, "gamma must be finite and non-negative");
    if (eps < 0.0 || eps > 1.0) return fail(h, NNP_ERR_ARG, "opt::algo::ADAM::read(Token&): Invalid eps.");
    cudaError_t ce = cudaSuccess;
    auto chk = [&](cudaError_t x) { if (x != cudaSuccess && ce == cudaSuccess) ce = x; };
    if (E.adam_master_stale) {
        // parameters in the reference packing: their wpar offsets, weight mask and FP64 values
        std::vector<int64_t> idx;
        std::vector<unsigned char> wm;
        pack_offsets(E, idx, &wm);
        std::vector<double> val;
        for (const auto &net : E.host.nets) {
            const int nl = (int)net.nodes.size() - 1;
            for (int l = 0; l < nl; ++l) val.insert(val.end(), net.b[l].begin(), net.b[l].end());
            for (int l = 0; l < nl; ++l) {
                const int ni = net.nodes[l], no = net.nodes[l + 1];
                for (int m = 0; m < ni; ++m)
                    for (int n = 0; n < no; ++n) val.push_back(net.w[l][(size_t)n * ni + m]);
            }
        }
        const bool fresh = E.adam_idx_host.size() != idx.size();
        E.adam_idx_host = idx;
        const size_t n = idx.size();
        chk(E.adam_wmask.reserve(n));
        chk(E.adam_idx.reserve(n));
        chk(E.adam_p.reserve(n));
        chk(E.adam_m.reserve(n));
        chk(E.adam_v.reserve(n));
        if (ce != cudaSuccess) return fail(h, NNP_ERR_CUDA, std::string("device allocation failed: ") + cudaGetErrorString(ce));
        chk(cudaMemcpyAsync(E.adam_idx.p, idx.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice, E.stream));
        chk(cudaMemcpyAsync(E.adam_p.p, val.data(), sizeof(double) * n, cudaMemcpyHostToDevice, E.stream));
        chk(cudaMemcpyAsync(E.adam_wmask.p, wm.data(), n, cudaMemcpyHostToDevice, E.stream));
        if (fresh) {        // first step (ADAM::resize): zero averages, powers beta^1
            chk(cudaMemsetAsync(E.adam_m.p, 0, sizeof(double) * n, E.stream));
            chk(cudaMemsetAsync(E.adam_v.p, 0, sizeof(double) * n, E.stream));
            E.adam_b1i = 0.9;
            E.adam_b2i = 0.999;
        }
        chk(cudaStreamSynchronize(E.stream));
        if (ce != cudaSuccess) return fail(h, NNP_ERR_CUDA, std::string("ADAM set-up failed: ") + cudaGetErrorString(ce));
        E.adam_master_stale = false;
    }
    std::string msg = nnp::run_adam(E, gamma, eps, reg, eta);
    if (!msg.empty()) return fail(h, NNP_ERR_CUDA, msg);
    // the host model is brought up to date when it is next read (host_params)
    E.host_stale = true;
    E.grad_valid = false;
    return NNP_OK;
}
}  // namespace

extern "C" {

int nnp_opt_reset(nnp_handle *h)
{
    if (!h) return NNP_ERR_ARG;
    h->E.adam_idx_host.clear();
    h->E.adam_master_stale = true;
    return NNP_OK;
}

int nnp_set_mma_wait(nnp_handle *h, int64_t polls)
{
    if (!h) return NNP_ERR_ARG;
    if (polls < 0 || polls > 0xffffffffll) return fail(h, NNP_ERR_ARG, "polls must be in [0, 2^32)");
    h->E.mma_wait_polls = (uint32_t)polls;
    h->E.graph_release();       // a captured step holds the old bound
    return NNP_OK;
}

int nnp_set_autotune(nnp_handle *h, int32_t enable)
{
    if (!h) return NNP_ERR_ARG;
    h->E.autotune = enable != 0;
    return NNP_OK;
}

int nnp_tune_params(const nnp_handle *h, int32_t *params, int32_t n, int32_t *source, const char **log)
{
    if (!h || (n > 0 && !params) || n < 0) return NNP_ERR_ARG;
    const nnp::TuneParams &p = h->E.tune;
    const int32_t v[5] = {p.symm_minb, p.force_minb, p.force_unroll, p.force_chunk, p.tc_per_sm};
    for (int k = 0; k < n && k < 5; ++k) params[k] = v[k];
    if (source) *source = h->E.tune_source;
    if (log) *log = h->E.tune_log.c_str();
    return NNP_OK;
}

int nnp_tune_cache_key(const char *potential_path, const char *device_name, int32_t n_sm, int32_t cap, char *key,
                       int32_t key_len)
{
    if (!potential_path || !device_name || !key || key_len <= 0 || n_sm <= 0 || cap <= 0) return NNP_ERR_ARG;
    std::string text;
    if (!read_file(potential_path, text)) return NNP_ERR_IO;
    nnp::Engine E;
    if (!nnp::read_potential(text, E.host).empty()) return NNP_ERR_PARSE;
    if (!E.build_tables().empty()) return NNP_ERR_UNSUPPORTED;
    const std::string k = nnp::tune_key(E, device_name, n_sm, cap);
    if ((int32_t)k.size() + 1 > key_len) return NNP_ERR_CAPACITY;
    std::memcpy(key, k.c_str(), k.size() + 1);
    return NNP_OK;
}

int nnp_tune_cache_store(const char *key, const int32_t *params, int32_t n)
{
    if (!key || !params || n != 5) return NNP_ERR_ARG;
    nnp::TuneParams p;
    p.symm_minb = params[0];
    p.force_minb = params[1];
    p.force_unroll = params[2];
    p.force_chunk = params[3];
    p.tc_per_sm = params[4];
    if (!nnp::tune_params_valid(p)) return NNP_ERR_ARG;
    return nnp::tune_cache_store(key, p) ? NNP_OK : NNP_ERR_IO;
}

int nnp_tune_cache_load(const char *key, int32_t *params, int32_t n)
{
    if (!key || !params || n != 5) return NNP_ERR_ARG;
    nnp::TuneParams p;
    if (!nnp::tune_cache_load(key, p)) return NNP_ERR_IO;
    const int32_t v[5] = {p.symm_minb, p.force_minb, p.force_unroll, p.force_chunk, p.tc_per_sm};
    for (int k = 0; k < 5; ++k) params[k] = v[k];
    return NNP_OK;
}

int nnp_set_loss(nnp_handle *h, int32_t kind, double delta)
{
    if (!h) return NNP_ERR_ARG;
    if (kind < NNP_LOSS_MSE || kind > NNP_LOSS_ASINH) return fail(h, NNP_ERR_ARG, "Invalid loss.");
    if ((kind == NNP_LOSS_HUBER || kind == NNP_LOSS_ASINH) && !(delta > 0.0 && std::isfinite(delta)))
        return fail(h, NNP_ERR_ARG, "the loss width delta must be positive and finite");
    h->E.loss_kind = kind;
    h->E.loss_delta = delta;
    return NNP_OK;
}

int nnp_train_grad(nnp_handle *h, const nnp_batch *batch, const double *e_ref, const double *f_ref, double w_f,
                   int32_t norm_mode, double *loss, double *grad, double *e_out, double *f_out, uint32_t flags)
{
    if (!h || !batch) return NNP_ERR_ARG;
    nnp::Engine &E = h->E;
    if (flags & ~(uint32_t)NNP_DEVICE_PTRS) return fail(h, NNP_ERR_ARG, "flags other than NNP_DEVICE_PTRS");
    const bool devp = (flags & NNP_DEVICE_PTRS) != 0;
    if (!e_ref || !loss) return fail(h, NNP_ERR_ARG, "e_ref and loss are required");
    if (!grad && !devp) return fail(h, NNP_ERR_ARG, "grad is required with host pointers");
    if (w_f != 0.0 && !f_ref) return fail(h, NNP_ERR_ARG, "f_ref is required when w_f is nonzero");
    if (!(w_f >= 0.0)) return fail(h, NNP_ERR_ARG, "w_f must be non-negative");
    if (norm_mode < 0 || norm_mode > 4) return fail(h, NNP_ERR_ARG, "unknown norm mode");
    const int S = batch->n_struct;
    if (S <= 0) return fail(h, NNP_ERR_ARG, "empty batch");
    if (w_f != 0.0)
        for (const auto &net : E.host.nets)
            if (net.neuron != nnp::NEU_LINEAR && net.neuron != nnp::NEU_SIGMOID && net.neuron != nnp::NEU_TANH)
                return fail(h, NNP_ERR_UNSUPPORTED, "the force term needs f'' of the activation (LINEAR, SIGMOID or TANH)");
    E.grad_valid = false;
    // forward: energies (no vacuum terms, as nnptefr subtracts them from the
    // labels) and forces, kept in the handle's buffers; the gradient kernels
    // run the FP32 networks, so the forward pass does too
    const int prec = E.precision;
    E.precision = NNP_PREC_FP32;
    int rc = compute_impl(h, batch, nullptr, nullptr, nullptr, nullptr, nullptr,
                          NNP_ENERGY | NNP_FORCES | KEEP_ON_DEVICE | (devp ? NNP_DEVICE_PTRS : 0u));
    E.precision = prec;
    if (rc != NNP_OK) return rc;
    const int64_t N = E.n_atoms;
    cudaError_t ce = cudaSuccess;
    auto chk = [&](cudaError_t x) { if (x != cudaSuccess && ce == cudaSuccess) ce = x; };
    chk(E.gE.reserve(std::max<int64_t>(N, 1)));
    chk(E.pgrad.reserve(E.wfloats));
    chk(E.loss_part.reserve(S + 1));
    chk(E.tvec.reserve(std::max<int64_t>(N, 1)));
    if (w_f != 0.0) chk(E.tang.reserve((size_t)std::max<int64_t>(N, 1) * E.gstride));
    if (!devp) chk(E.train_ref.reserve(S + 3 * (size_t)std::max<int64_t>(N, 1)));
    if (E.pack_n == 0) {
        std::vector<int64_t> idx;
        pack_offsets(E, idx, nullptr);
        chk(E.pack_idx.reserve(idx.size()));
        chk(E.grad_pack.reserve(idx.size()));
        if (ce == cudaSuccess)
            chk(cudaMemcpyAsync(E.pack_idx.p, idx.data(), sizeof(int64_t) * idx.size(), cudaMemcpyHostToDevice, E.stream));
        E.pack_n = (int64_t)idx.size();
    }
    if (ce != cudaSuccess) return fail(h, NNP_ERR_CUDA, std::string("device allocation failed: ") + cudaGetErrorString(ce));
    // labels on the device
    const double *er = e_ref, *fr = f_ref;
    if (!devp) {
        chk(cudaMemcpyAsync(E.train_ref.p, e_ref, sizeof(double) * S, cudaMemcpyHostToDevice, E.stream));
        if (w_f != 0.0)
            chk(cudaMemcpyAsync(E.train_ref.p + S, f_ref, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, E.stream));
        er = E.train_ref.p;
        fr = E.train_ref.p + S;
    }
    if (ce != cudaSuccess) return fail(h, NNP_ERR_CUDA, std::string("copy failed: ") + cudaGetErrorString(ce));
    // loss and the per-atom factors on the device (nnptefr.cpp:1331-1380)
    const int64_t *off = devp ? batch->atom_off : E.atom_off.p;
    std::string msg = nnp::run_train_loss(E, off, er, fr, w_f, norm_mode, E.loss_part.p + S);
    if (!msg.empty()) return fail(h, NNP_ERR_CUDA, msg);
    // gradient kernels; with device pointers the batch's types are the caller's array
    int *own_type = E.type.p;
    if (devp) E.type.p = const_cast<int32_t *>(batch->type);
    msg = nnp::run_train_grad(E, w_f != 0.0);
    E.type.p = own_type;
    if (!msg.empty()) return fail(h, NNP_ERR_CUDA, msg);
    E.grad_valid = true;
    if (devp) {
        chk(cudaMemcpyAsync(loss, E.loss_part.p + S, sizeof(double), cudaMemcpyDeviceToDevice, E.stream));
        if (grad) {
            msg = nnp::run_gather_grad(E, E.pack_idx.p, E.pack_n, grad);
            if (!msg.empty()) return fail(h, NNP_ERR_CUDA, msg);
        }
        if (e_out) chk(cudaMemcpyAsync(e_out, E.e_struct.p, sizeof(double) * S, cudaMemcpyDeviceToDevice, E.stream));
        if (f_out) chk(cudaMemcpyAsync(f_out, E.force.p, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, E.stream));
        if (ce != cudaSuccess) return fail(h, NNP_ERR_CUDA, std::string("output copy failed: ") + cudaGetErrorString(ce));
        return NNP_OK;
    }
    msg = nnp::run_gather_grad(E, E.pack_idx.p, E.pack_n, E.grad_pack.p);
    if (!msg.empty()) return fail(h, NNP_ERR_CUDA, msg);
    chk(cudaMemcpyAsync(loss, E.loss_part.p + S, sizeof(double), cudaMemcpyDeviceToHost, E.stream));
    chk(cudaMemcpyAsync(grad, E.grad_pack.p, sizeof(double) * E.pack_n, cudaMemcpyDeviceToHost, E.stream));
    if (e_out) chk(cudaMemcpyAsync(e_out, E.e_struct.p, sizeof(double) * S, cudaMemcpyDeviceToHost, E.stream));
    if (f_out) chk(cudaMemcpyAsync(f_out, E.force.p, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, E.stream));
    chk(cudaStreamSynchronize(E.stream));
    if (ce != cudaSuccess) return fail(h, NNP_ERR_CUDA, std::string("gradient failed: ") + cudaGetErrorString(ce));
    return NNP_OK;
}

}  // extern "C"
