// nnp_tune.cpp -- autotuner of the per-atom kernels' launch and tile choices.
//
// The specialised symmetry-function and force kernels are compiled with
// register budgets (resident blocks per SM), a pair-loop unroll factor and a
// coefficient chunk size (TuneParams, nnp_engine.h); the tensor-core network
// kernel runs a number of CTAs per SM.  Which values are fastest depends on
// the potential (block sizes, damping groups, network widths), on the
// neighbour counts of the workload and on the GPU.  On the first call of a
// neighbour-capacity class the tuner compiles a small set of candidates (in
// parallel host threads; NVRTC), times each on the caller's own batch with
// the library's CUDA-event stage timers, keeps the fastest value of each
// kernel's choices independently (each choice affects one kernel only), and
// stores the result in the tuning cache beside the compiled-kernel cache,
// keyed by the potential, the GPU and the capacity class.  Later handles of
// the same potential on the same GPU load it without timing anything.
//
// No reference counterpart: the reference runs on the CPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <thread>
#include <unistd.h>
#include <vector>

#include "../../include/nnp_b200.h"
#include "nnp_engine.h"

namespace nnp {

namespace {

// Candidate values of each choice.  Candidate k of the tuning run uses
// option k of every list (the last option when a list is shorter), so every
// option of every list is timed once with as few compilations as the longest
// list: the symmetry-function options only change k_symm_jit, the force
// options only k_force_jit, the network option only k_nn_tc.
struct ForceOpt { int minb, unroll, chunk; };
const int kSymmMinb[] = {4, 3, 2};
const ForceOpt kForce[] = {{1, 1, NNP_PCH}, {2, 1, NNP_PCH}, {1, 1, 192}, {2, 1, 192}, {2, 1, 144}};
const int kTcPerSm[] = {0, 1, 2, 3};
constexpr int kCandidates = 5;
constexpr int kReps = 3;        // timed repetitions per candidate (median)

template <class T, size_t N>
const T &pick(const T (&a)[N], int k) { return a[std::min<size_t>((size_t)k, N - 1)]; }

TuneParams candidate(int k)
{
    TuneParams p;
    p.symm_minb = pick(kSymmMinb, k);
    const ForceOpt &f = pick(kForce, k);
    p.force_minb = f.minb;
    p.force_unroll = f.unroll;
    p.force_chunk = f.chunk;
    p.tc_per_sm = pick(kTcPerSm, k);
    return p;
}

// capacity class of a neighbour capacity: 64, 128, 256 slots (the largest
// class the device path stages is NNP_MAX_NBR)
int cap_class(int cap)
{
    int c = 64;
    while (c < cap && c < NNP_MAX_NBR) c <<= 1;
    return c;
}

std::string tune_file()
{
    const std::string d = cache_dir();
    return d.empty() ? "" : d + "/tuning.txt";
}

std::string params_text(const TuneParams &p)
{
    char b[160];
    std::snprintf(b, sizeof b, "symm_minb=%d force_minb=%d force_unroll=%d force_chunk=%d tc_per_sm=%d",
                  p.symm_minb, p.force_minb, p.force_unroll, p.force_chunk, p.tc_per_sm);
    return b;
}

}  // namespace

bool tune_params_valid(const TuneParams &q)
{
    return q.symm_minb >= 1 && q.symm_minb <= 4 && q.force_minb >= 1 && q.force_minb <= 4 && q.force_unroll >= 1 &&
           q.force_unroll <= 4 && q.force_chunk >= 8 && q.force_chunk <= NNP_PCH && q.tc_per_sm >= 0 &&
           q.tc_per_sm <= 4;
}

bool tune_needed(const Engine &E, int cap)
{
    return std::find(E.tuned_caps.begin(), E.tuned_caps.end(), cap_class(cap)) == E.tuned_caps.end();
}

namespace {

bool parse_params(const std::string &text, TuneParams &p)
{
    TuneParams q;
    int seen = 0;
    std::istringstream is(text);
    std::string tok;
    while (is >> tok) {
        const size_t eq = tok.find('=');
        if (eq == std::string::npos) return false;
        const std::string k = tok.substr(0, eq);
        char *end = nullptr;
        const long v = std::strtol(tok.c_str() + eq + 1, &end, 10);
        if (!end || *end) return false;
        if (k == "symm_minb") q.symm_minb = (int)v, seen |= 1;
        else if (k == "force_minb") q.force_minb = (int)v, seen |= 2;
        else if (k == "force_unroll") q.force_unroll = (int)v, seen |= 4;
        else if (k == "force_chunk") q.force_chunk = (int)v, seen |= 8;
        else if (k == "tc_per_sm") q.tc_per_sm = (int)v, seen |= 16;
        else return false;
    }
    const bool ok = seen == 31 && tune_params_valid(q);
    if (ok) p = q;
    return ok;
}

float median3(std::vector<float> v)
{
    std::sort(v.begin(), v.end());
    return v.empty() ? 0.f : v[v.size() / 2];
}

}  // namespace

// Environment overrides of the defaults (experiments and tests):
// NNP_SYMM_MINB, NNP_FORCE_MINB, NNP_FORCE_UNROLL (1..4), NNP_FORCE_CHUNK
// (1..NNP_PCH).
void tune_from_env(TuneParams &p)
{
    auto knob = [](const char *name, int lo, int hi, int &v) {
        const char *s = std::getenv(name);
        if (!s || !s[0]) return;
        const int b = std::atoi(s);
        if (b >= lo && b <= hi) v = b;
    };
    knob("NNP_SYMM_MINB", 1, 4, p.symm_minb);
    knob("NNP_FORCE_MINB", 1, 4, p.force_minb);
    knob("NNP_FORCE_UNROLL", 1, 4, p.force_unroll);
    knob("NNP_FORCE_CHUNK", 1, NNP_PCH, p.force_chunk);
}

// Key of one tuning: the specialised source at the default choices (it holds
// every basis parameter and the kernel code), the network shapes, the
// device's name and SM count, and the capacity class.
std::string tune_key(const Engine &E, const std::string &device, int nsm, int cap)
{
    std::ostringstream os;
    os << jit_source(E, TuneParams());
    for (int t = 0; t < E.dpot.ntypes; ++t) {
        os << "|net";
        for (int l = 0; l <= E.dpot.t[t].nlayer; ++l) os << ' ' << E.dpot.t[t].nodes[l];
    }
    os << "|prec " << E.precision;
    char b[96];
    std::snprintf(b, sizeof b, "%016llx", (unsigned long long)source_hash(os.str()));
    std::string dev = device;
    for (char &c : dev)
        if (c == ' ' || c == '\t' || c == '\n') c = '_';
    return std::string(b) + ":" + dev + ":" + std::to_string(nsm) + ":cap" + std::to_string(cap_class(cap));
}

// One line per key in the tuning file: "<key> <params>"; the last line of a
// key wins.  Malformed lines are skipped.
bool tune_cache_load(const std::string &key, TuneParams &p)
{
    const std::string f = tune_file();
    if (f.empty()) return false;
    std::ifstream in(f);
    std::string line;
    bool found = false;
    while (std::getline(in, line)) {
        const size_t sp = line.find(' ');
        if (sp == std::string::npos || line.compare(0, sp, key) != 0 || sp != key.size()) continue;
        TuneParams q;
        if (parse_params(line.substr(sp + 1), q)) {
            p = q;
            found = true;
        }
    }
    return found;
}

bool tune_cache_store(const std::string &key, const TuneParams &p)
{
    const std::string f = tune_file();
    if (f.empty()) return false;
    const std::string dir = f.substr(0, f.rfind('/'));
    for (size_t k = 1; k <= dir.size(); ++k)
        if (k == dir.size() || dir[k] == '/') mkdir(dir.substr(0, k).c_str(), 0755);
    std::ofstream out(f, std::ios::app);
    if (!out) return false;
    out << key << ' ' << params_text(p) << '\n';   // one write of one line: appends from several processes interleave by line
    return (bool)out;
}

// Tunes the handle for capacity `cap` on the batch run_step computes (the
// device-side step of nnp_compute; it runs eagerly here, stage timers on).
// Leaves the best choices compiled and loaded in E.  Returns "" or an error.
std::string autotune(Engine &E, int cap, const std::function<std::string()> &run_step)
{
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceProp prop;
    std::memset(&prop, 0, sizeof prop);
    cudaGetDeviceProperties(&prop, dev);
    const std::string key = tune_key(E, prop.name, nsm, cap);
    const int cls = cap_class(cap);
    E.tuned_caps.push_back(cls);
    TuneParams best;
    if (tune_cache_load(key, best)) {
        if (!(best == E.tune)) {
            const TuneParams old = E.tune;
            E.tune = best;
            std::string msg = jit_build(E);
            if (!msg.empty()) {
                E.tune = old;
                jit_build(E);
                return msg;
            }
        }
        E.tune_source = 1;
        E.tune_log = "loaded " + key + " " + params_text(best);
        return "";
    }
    // compile every candidate (NVRTC; in parallel, results land in the caches)
    std::vector<TuneParams> cand;
    for (int k = 0; k < kCandidates; ++k) cand.push_back(candidate(k));
    {
        std::vector<std::thread> th;
        std::vector<std::string> errs(cand.size());
        for (size_t k = 0; k < cand.size(); ++k)
            th.emplace_back([&, k] {
                std::string src;
                std::vector<char> cubin;
                errs[k] = jit_compile_params(E, cand[k], src, cubin);
            });
        for (auto &t : th) t.join();
        for (const auto &e : errs)
            if (!e.empty()) return "autotune: " + e;
    }
    const bool timing = E.timing;
    const TuneParams start = E.tune;
    if (!E.ev[0])
        for (auto &e : E.ev)
            if (cudaEventCreate(&e) != cudaSuccess) return "autotune: cudaEventCreate failed";
    E.timing = true;
    std::vector<float> t_symm(cand.size()), t_nn(cand.size()), t_force(cand.size());
    std::string err;
    for (size_t k = 0; k < cand.size() && err.empty(); ++k) {
        E.tune = cand[k];
        err = jit_build(E);
        std::vector<float> s, n, f;
        for (int r = 0; r < kReps + 1 && err.empty(); ++r) {
            err = run_step();
            if (!err.empty()) break;
            if (cudaStreamSynchronize(E.stream) != cudaSuccess) {
                err = std::string("autotune: ") + cudaGetErrorString(cudaGetLastError());
                break;
            }
            if (r == 0) continue;               // the first run of a candidate warms its caches
            float ms[3] = {0.f, 0.f, 0.f};
            for (int q = 0; q < 3; ++q)
                if (cudaEventElapsedTime(&ms[q], E.ev[q + 1], E.ev[q + 2]) != cudaSuccess) cudaGetLastError();
            s.push_back(ms[0]);
            n.push_back(ms[1]);
            f.push_back(ms[2]);
        }
        t_symm[k] = median3(s);
        t_nn[k] = median3(n);
        t_force[k] = median3(f);
    }
    E.timing = timing;
    if (!err.empty()) {
        E.tune = start;
        jit_build(E);
        return err;
    }
    // the fastest value of each kernel's choices
    size_t ks = 0, kn = 0, kf = 0;
    for (size_t k = 1; k < cand.size(); ++k) {
        if (t_symm[k] < t_symm[ks]) ks = k;
        if (t_nn[k] < t_nn[kn]) kn = k;
        if (t_force[k] < t_force[kf]) kf = k;
    }
    best.symm_minb = cand[ks].symm_minb;
    best.force_minb = cand[kf].force_minb;
    best.force_unroll = cand[kf].force_unroll;
    best.force_chunk = cand[kf].force_chunk;
    // the network choice only matters for the tensor-core kernel
    best.tc_per_sm = E.precision == NNP_PREC_FP32 ? start.tc_per_sm : cand[kn].tc_per_sm;
    E.tune = best;
    std::string msg = jit_build(E);
    if (!msg.empty()) {
        E.tune = start;
        jit_build(E);
        return msg;
    }
    tune_cache_store(key, best);
    std::ostringstream log;
    log << "tuned " << key << " " << params_text(best) << "; ms (symm, networks, forces) per candidate:";
    for (size_t k = 0; k < cand.size(); ++k) {
        char b[96];
        std::snprintf(b, sizeof b, " [%.3f %.3f %.3f]", t_symm[k], t_nn[k], t_force[k]);
        log << b;
    }
    E.tune_source = 2;
    E.tune_log = log.str();
    return "";
}

}  // namespace nnp
