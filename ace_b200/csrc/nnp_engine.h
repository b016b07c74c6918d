// nnp_engine.h -- device buffers of one handle and the launch sequence of the
// energy/force path.  Used by the C ABI (nnp_api.cu); kernels live in
// nnp_kernels.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <string>
#include <vector>

#include "nnp_internal.h"

namespace nnp {

// per-structure neighbour-search grid (filled on the device)
struct StructGrid {
    double R[9];      // R[3n+d]: component d of lattice vector n
    double B[9];      // B[3n+d]: reciprocal row n (fractional coordinate n = B_n . x)
    int nc[3];        // cells per lattice direction
    int m[3];         // cells searched on each side
    int cell_base;    // first global cell index of this structure
    int pbc;
};

template <class T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    cudaError_t reserve(size_t count)
    {
        if (count <= n) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        size_t c = count + count / 4 + 16;
        cudaError_t e = cudaMalloc((void **)&p, c * sizeof(T));
        if (e == cudaSuccess) n = c;
        return e;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

// Launch and tile choices of the per-atom kernels.  Defaults are the values
// measured best on the batched workload; the autotuner (nnp_tune.cpp) times
// alternatives on the caller's data and replaces them.
struct TuneParams {
    int symm_minb = 4;          // blocks per SM the specialised symmetry-function kernel's registers are budgeted for (1..4)
    int force_minb = 1;         // the same for the specialised force kernel (1..4)
    int force_unroll = 1;       // unroll factor of the specialised force kernel's pair loop (1..4)
    int force_chunk = NNP_PCH;  // pair coefficients per chunk of the force kernel (8..NNP_PCH); sets its shared memory
    int tc_per_sm = 0;          // CTAs per SM of the tensor-core network kernel (0: as many as fit, at most 4)
    bool operator==(const TuneParams &o) const
    {
        return symm_minb == o.symm_minb && force_minb == o.force_minb && force_unroll == o.force_unroll &&
               force_chunk == o.force_chunk && tc_per_sm == o.tc_per_sm;
    }
};

struct Engine {
    // potential
    HostPot host;
    DevPot dpot{};
    DevPot *d_pot = nullptr;
    DBuf<float2> rpar;            // radial (rs, eta)
    DBuf<float4> apar;            // angular (lambdaf, zeta, ieta2, damp | izeta << 8)
    DBuf<float> wpar;             // networks, FP32 (layout in nnp_internal.h)
    DBuf<double> vac;             // per-type vacuum energies
    int64_t wfloats = 0;
    int gstride = 0;              // row length of G / dE/dG (max n_input rounded up to 4)
    int precision = 0;
    uint32_t mma_wait_polls = 0;  // bound of one tensor-core MMA-chain wait (0: the kernel's default)
    bool acc64 = false;           // FP64 running sums of the symmetry functions
    bool symm64 = false;          // symmetry functions evaluated in FP64 (k_symm_f64)
    DBuf<double2> rpar64;         // radial (rs, eta) in FP64
    DBuf<double4> apar64;         // angular (lambda/2, zeta, 1/eta_run^2, 0) in FP64
    DBuf<double> cut64;           // rc of every distinct cutoff in FP64
    std::vector<double2> rpar64_host;
    std::vector<double4> apar64_host;
    std::vector<double> cut64_host;
    std::vector<float2> rpar_host;
    std::vector<float4> apar_host;
    std::vector<float> wpar_host;
    std::vector<double> vac_host;

    // kernels specialised for this potential at run time (nnp_jit.cpp)
    TuneParams tune;              // launch / tile choices the specialised kernels are compiled with
    bool autotune = false;        // tune on the first call of each neighbour-capacity class (nnp_set_autotune)
    std::vector<int> tuned_caps;  // capacity classes already tuned (or loaded from the cache) by this handle
    int tune_source = 0;          // 0 defaults, 1 loaded from the tuning cache, 2 tuned on this handle's data
    std::string tune_log;         // the last tuning's measurements
    bool use_jit = true;
    void *jit_module = nullptr;   // cudaLibrary_t
    void *jit_symm = nullptr, *jit_force = nullptr, *jit_tangent = nullptr;   // cudaKernel_t
    std::string jit_source, jit_error;

    // stream / events
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    // batch
    int n_struct = 0;
    int64_t n_atoms = 0;
    int64_t n_ghost = 0;          // the last n_ghost atoms are ghosts: neighbours only (nnp_compute_local_ghost)
    int64_t n_centre = 0;         // n_atoms - n_ghost: atoms that are centres (own an energy and symmetry functions)
    int cap = 0;                  // neighbour slots per atom
    int tot_cells = 0;
    DBuf<int64_t> atom_off;
    DBuf<double> pos, cell, xw;
    DBuf<int> type, atom_struct, atom_cell;
    DBuf<StructGrid> grid;
    DBuf<double> bbox;            // bounding box of each free structure [6 * S]
    DBuf<int> cell_cnt, cell_start, cell_fill, cell_atoms, scan_tmp;
    DBuf<int> cell_tcnt;          // members of each type per cell [cell][type]
    DBuf<double4> cell_pos;       // cell-ordered wrapped positions, type in .w
    DBuf<int> order;              // atoms grouped by element (visiting order of the per-atom kernels)
    DBuf<int> type_fill;          // [2 * (NNP_MAX_TYPES + 1) + 1] element counts (out-of-range types last), fill cursors, neighbour-search work items
    DBuf<int4> neigh_items;       // neighbour-search work items {cell, structure, first atom, end atom}
    DBuf<float4> nbr;
    DBuf<int> nbr_cnt;
    DBuf<float> G, dEdG, e_atom;
    DBuf<double> e_struct, force, symm_d;
    DBuf<DevErr> err;
    DBuf<double> vir;             // per-structure virial [9 * S] (when want_virial)
    DBuf<double> eatom_d;         // per-atom energies for host-pointer calls
    bool want_virial = false;
    // training (nnp_train_grad)
    DBuf<float4> tvec;            // per-atom force factor V_i (x, y, z, 0)
    DBuf<float> gE;               // per-atom energy factor
    DBuf<float> tang;             // tangent symmetry functions C [N * gstride]
    DBuf<double> pgrad;           // parameter gradient in the wpar layout [wfloats]
    bool grad_valid = false;      // pgrad holds the gradient of the last nnp_train_grad
    DBuf<double> loss_part;       // per-structure loss terms [S + 1] (the last entry: the batch loss)
    DBuf<double> train_ref;       // device copies of host labels: e_ref [S], f_ref [3N]
    DBuf<double> grad_pack;       // gradient in the reference packing (host-pointer calls)
    DBuf<int64_t> pack_idx;       // wpar offset of every parameter in the reference packing
    int64_t pack_n = 0;
    // ADAM state (nnp_opt_adam): wpar offsets of the parameters in the
    // reference packing, FP64 master copy and running averages
    std::vector<int64_t> adam_idx_host;
    DBuf<int64_t> adam_idx;
    DBuf<double> adam_p, adam_m, adam_v;
    DBuf<unsigned char> adam_wmask;   // 1 for a weight, 0 for a bias (the weight-decay mask)
    double adam_b1i = 0.9, adam_b2i = 0.999;
    bool adam_master_stale = true;  // the master copy must be reloaded from the host model
    bool host_stale = false;        // the host model lags the master copy (device optimiser steps)
    int loss_kind = 1;            // energy-loss kind of nnp_train_grad (NNP_LOSS_*)
    double loss_delta = 1.0;      // its width (HUBER, ASINH)
    float *noalloc_e_atom = nullptr;  // device address of the allocation-free call's scratch (looked up once)
    DevErr *h_err = nullptr;      // pinned
    // pinned staging for host-pointer calls
    void *h_stage = nullptr;
    size_t h_stage_bytes = 0;

    std::string last_error;

    // stage timers and launch counter
    bool timing = false;

    // CUDA graph of the device-side step, replayed while the call's shape and
    // device pointers repeat (see graph_key in nnp_api.cu)
    bool use_graphs = true;
    void *graph_exec = nullptr;     // cudaGraphExec_t
    std::vector<int64_t> graph_key;
    int64_t graph_launches = 0;     // kernels in the graph
    void graph_release();
    cudaEvent_t ev[6] = {};
    int64_t launches = 0;
    void mark(int k)
    {
        if (timing && ev[k]) cudaEventRecord(ev[k], stream);
    }

    // device tables of the potential from `host` (host-side only), and their upload
    std::string build_tables();
    std::string upload();
    void free_all();
};

// launch sequence (nnp_kernels.cu); each returns "" or an error message
std::string run_prepare(Engine &E, int64_t n_atoms, int n_struct, int pbc);
std::string run_neighbors(Engine &E, int pbc);
std::string run_symm(Engine &E);
std::string run_nn(Engine &E);
std::string run_force(Engine &E);
std::string run_energy(Engine &E, bool vacuum);
std::string run_symm_to_double(Engine &E, double *out);
std::string run_atom_energy(Engine &E, bool vacuum, double *out);
std::string run_nn_from_symm(Engine &E, const double *symm_d, int gstride_in);
std::string run_neighbor_counts(Engine &E, int *d_counts);
std::string run_train_grad(Engine &E, bool with_force);
std::string run_adam(Engine &E, double gamma, double eps, int reg, double eta);
std::string run_train_loss(Engine &E, const int64_t *off, const double *e_ref, const double *f_ref, double w_f,
                           int norm_mode, double *loss_dev);
std::string run_gather_grad(Engine &E, const int64_t *idx, int64_t n, double *out);
std::string run_input_stats(Engine &E, std::vector<int64_t> &count, std::vector<double> &stats);
std::string taylor_expand(int S, const int64_t *atom_off, const double *pos, const double *energy,
                          const double *forces, int nadd, int dist, double rdelta, uint64_t seed,
                          std::vector<int64_t> &out_off, std::vector<int> &out_src, std::vector<double> &out_pos,
                          std::vector<double> &out_energy);
int tc_smem_bytes(const Engine &E, bool split);     // 0: networks do not fit the tensor-core path
std::string run_nn_tc(Engine &E, bool split);
std::string run_energy_symm_noalloc(Engine &E, int S, int64_t N, const int64_t *off, const int *type,
                                    const float *G, int gstride, bool vacuum, double *energy);

// autotuner (nnp_tune.cpp): key of the tuning cache and the tuning itself,
// which calls run_step (the device-side step, stage timers on) per candidate
std::string tune_key(const Engine &E, const std::string &device, int nsm, int cap);
bool tune_cache_load(const std::string &key, TuneParams &p);
bool tune_cache_store(const std::string &key, const TuneParams &p);
std::string autotune(Engine &E, int cap, const std::function<std::string()> &run_step);
bool tune_needed(const Engine &E, int cap);
bool tune_params_valid(const TuneParams &p);
void tune_from_env(TuneParams &p);

// run-time specialised kernels (nnp_jit.cpp)
std::string jit_compile(const Engine &E, std::string &source, std::vector<char> &cubin);
std::string jit_compile_params(const Engine &E, const TuneParams &tp, std::string &source, std::vector<char> &cubin);
std::string jit_source(const Engine &E, const TuneParams &p);
uint64_t source_hash(const std::string &s);
std::string cache_dir();
std::string jit_build(Engine &E);
std::string &jit_last_log();   // compiler messages of the last NVRTC compilation
void jit_release(Engine &E);
std::string jit_launch(void *fn, int grid, int block, size_t smem, cudaStream_t stream, void **args);

}  // namespace nnp
