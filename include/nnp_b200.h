/*
 * nnp_b200.h -- C ABI of the B200 NNP energy/force library (libnnp_b200.so).
 *
 * This is the drop-in boundary for the Behler-Parrinello NNP hot path of the
 * reference (markdellostritto/ace): neighbour list -> radial/angular symmetry
 * functions -> per-element atomic networks -> analytic forces, plus the
 * weight gradient of the energy(+force) training loss.  Each entry point names
 * the reference interface it replaces (paths inside the reference's src/).
 *
 * Conventions
 *  - Every function returns an int status: NNP_OK (0) or a negative NNP_ERR_*
 *    code; nothing throws across the ABI.  nnp_last_error() gives the message.
 *  - A handle owns its device memory and one CUDA stream; it is not shared
 *    between host threads.  Device buffers grow monotonically.
 *  - Positions, cells and outputs are FP64 on the host side; the device path
 *    computes in FP32 (or BF16 network layers) with FP64 accumulation of forces
 *    and per-structure energies.
 *  - Structures are passed as a CSR batch (nnp_batch).  Atom types are NNP
 *    type indices (nnp_type_index), i.e. the reference's map_ (nnp.hpp:68).
 */
#ifndef NNP_B200_H
#define NNP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define NNP_OK 0
#define NNP_ERR_ARG (-1)          /* bad argument (null pointer, bad size, bad flag)      */
#define NNP_ERR_IO (-2)           /* file could not be opened                             */
#define NNP_ERR_PARSE (-3)        /* potential / basis file malformed                     */
#define NNP_ERR_CUDA (-4)         /* CUDA runtime error                                   */
#define NNP_ERR_CAPACITY (-5)     /* an internal capacity was exceeded and could not grow */
#define NNP_ERR_UNSUPPORTED (-6)  /* a feature the device path does not implement         */
#define NNP_ERR_TYPE (-7)         /* atom type index out of range                         */
#define NNP_ERR_NOT_FINITE (-8)   /* a non-finite energy or force was produced            */

/* ---- precision of the atomic-network layers ---- */
#define NNP_PREC_FP32 0           /* FP32 CUDA-core network layers (plain path)                   */
#define NNP_PREC_BF16 1           /* BF16 tensor-core layers, FP32 accumulation (tcgen05, sm_100a) */
#define NNP_PREC_BF16X3 2         /* split-BF16 (hi/lo, 3 products) tensor-core layers            */

/* ---- nnp_compute flags ---- */
#define NNP_ENERGY 1u             /* write per-structure energies                                */
#define NNP_FORCES 2u             /* write forces                                                */
#define NNP_VACUUM 4u             /* add per-type vacuum energies (NNP::compute_energy semantics) */
#define NNP_DEVICE_PTRS 8u        /* every pointer in the batch and outputs is device memory     */
#define NNP_SYMM 16u              /* write the symmetry-function rows (symm_out)                 */

/* CSR batch of periodic (or free) structures.
 *  atom_off[n_struct+1]  atoms of structure s are [atom_off[s], atom_off[s+1])
 *  pos[3*N]              Cartesian positions, x y z per atom
 *  type[N]               NNP type index of each atom
 *  cell[9*n_struct]      lattice vectors of structure s: cell[9s+3n+d] is
 *                        component d of vector n, i.e. Cell::R (struc/cell.hpp:23,
 *                        lattice vectors as columns) stored column-major
 *  pbc                   nonzero: periodic in all three directions;
 *                        zero: free boundaries (cell ignored)                   */
typedef struct {
    int32_t n_struct;
    const int64_t *atom_off;
    const double *pos;
    const int32_t *type;
    const double *cell;
    int32_t pbc;
} nnp_batch;

typedef struct nnp_handle nnp_handle;

/* Reads a potential file; replaces NNP::read(const char*, NNP&) (src/nnp/nnp.cpp:181-190,
 * format nnp.cpp:243-307) and uploads it to the current CUDA device. */
int nnp_create_from_file(const char *potential_path, nnp_handle **out);

/* Builds a potential from its pieces the way nnptefr does (nnptefr.cpp:2023-2031):
 * type lines as in the potential file (nnh.cpp:65-93), the global cutoff, one
 * per-element basis file each (NNP::read_basis, nnp.cpp:96-156, written by
 * make_basis), and one network description per element given as a text block in
 * the ANN file format (ml/nn.cpp:1536-1613). */
int nnp_create_from_basis(int32_t ntypes, const char *const *type_lines, double rc,
                          const char *const *basis_paths, const char *const *network_texts,
                          nnp_handle **out);

/* Releases the handle and all its device memory. */
int nnp_destroy(nnp_handle *h);

/* Writes the potential; replaces NNP::write(const char*, const NNP&) (nnp.cpp:165-236). */
int nnp_write(const nnp_handle *h, const char *path);

/* Network-layer precision (NNP_PREC_*). */
int nnp_set_precision(nnp_handle *h, int32_t precision);

/* Bound of each wait of the tensor-core network kernel for one MMA chain, in
 * tests of its barrier (no reference counterpart; 0 = the default, ~2^26
 * tests, well above any chain's time).  A wait that runs out makes the call
 * return NNP_ERR_CUDA ("an MMA wait timed out") instead of hanging; the
 * kernel then waits for the chain in flight (default bound) and releases its
 * tensor memory, so the handle stays usable. */
int nnp_set_mma_wait(nnp_handle *h, int64_t polls);

/* Precision of the symmetry functions: NNP_ACC_FP32 (default) computes every
 * pair/triplet term and running sum in FP32; NNP_ACC_FP64 adds the FP32 terms
 * into FP64 sums (~sqrt(T/32) ulp less error for T triplets per atom);
 * NNP_SYMM_FP64 evaluates the terms themselves in FP64 (neighbour
 * displacements recovered in FP64 from the positions, FP64 basis functions
 * and parameters, prebuilt kernel), storing the rows as FP32.  Networks and
 * forces stay FP32 in every mode.  NNP_SYMM_FP64 is for potentials whose
 * input scaling (inpw) is large enough to turn the ~1e-7 relative FP32 error
 * of the terms into force errors above 1e-5 eV/A; it is several times slower. */
#define NNP_ACC_FP32 0
#define NNP_ACC_FP64 1
#define NNP_SYMM_FP64 2
int nnp_set_accumulation(nnp_handle *h, int32_t acc);

/* Kernels specialised for the loaded basis.  At creation the library writes
 * CUDA source in which every GAUSS angular block is straight-line code with its
 * parameters as literals and compiles it for sm_100a with NVRTC (environment
 * NNP_JIT=0 skips this).  enable=0 switches back to the prebuilt kernels;
 * nnp_specialization reports whether the specialised kernels are in use and
 * returns their source text. */
int nnp_set_specialization(nnp_handle *h, int32_t enable);
int nnp_specialization(const nnp_handle *h, int32_t *active, const char **source);

/* Writes and compiles the specialised kernels of a potential file without a GPU
 * (NVRTC only); log receives the generated source, or the compiler's message
 * when compilation fails (NNP_ERR_CUDA). */
int nnp_specialization_check(const char *potential_path, char *log, int32_t log_len);

/* Autotuning of the launch and tile choices of the per-atom kernels (no
 * reference counterpart; the reference runs on the CPU).  With enable = 1
 * (or NNP_AUTOTUNE=1 in the environment at creation), the first
 * energy+force call of each neighbour-capacity class (64, 128, 256 slots per
 * atom) looks the choice up in the tuning cache (NNP_CACHE_DIR, default
 * ~/.cache/nnp_b200, file tuning.txt), keyed by the potential, the network
 * shapes, the precision, the GPU and the class; without an entry it compiles
 * a few candidates and times each on that call's own batch (CUDA events),
 * keeps the fastest choice of each kernel, stores it, and then computes the
 * call's results with it.  The first such call therefore takes seconds
 * longer.  Results do not depend on the choices beyond FP32 summation order.
 * Choices (params[0..4]): blocks per SM the symmetry-function kernel's
 * registers are budgeted for, the same for the force kernel, the force
 * kernel's pair-loop unroll, its pair coefficients per chunk (a smaller
 * chunk needs less shared memory, so more blocks may be resident), and CTAs
 * per SM of the tensor-core network kernel (0 = as many as fit).
 * nnp_tune_params returns the handle's current choices, where they came from
 * (*source: 0 defaults, 1 tuning cache, 2 tuned on this handle) and the last
 * tuning's measurements (*log).  nnp_tune_cache_key / _store / _load read and
 * write the cache without a GPU (e.g. to seed it for a fleet of one GPU model):
 * key has room for key_len bytes (about 100 are needed). */
int nnp_set_autotune(nnp_handle *h, int32_t enable);
int nnp_tune_params(const nnp_handle *h, int32_t *params, int32_t n, int32_t *source, const char **log);
int nnp_tune_cache_key(const char *potential_path, const char *device_name, int32_t n_sm, int32_t cap, char *key,
                       int32_t key_len);
int nnp_tune_cache_store(const char *key, const int32_t *params, int32_t n);
int nnp_tune_cache_load(const char *key, int32_t *params, int32_t n);

/* Launch on this CUDA stream (cudaStream_t) instead of the handle's own one. */
int nnp_set_stream(nnp_handle *h, void *cuda_stream);

/* CUDA graphs (on by default; no reference counterpart, the reference runs on
 * the CPU).  The device-side step of nnp_compute / nnp_compute_md -- neighbour
 * list, symmetry functions, networks, forces, energies -- launches only
 * kernels whose sizes the host knows, so when a call repeats the previous
 * call's shape (atom and structure counts, flags, capacity, device buffers)
 * the library captures the step once and then replays it as one graph, as in
 * an MD loop.  Not used on the legacy default stream or with stage timers on. */
int nnp_set_graphs(nnp_handle *h, int32_t enable);

/* ---- inspection: NNP::ntypes / index / rc / NNH::nInput (nnp.hpp:78-87, nnh.hpp:140-142) ---- */
int nnp_ntypes(const nnp_handle *h, int32_t *ntypes);
int nnp_type_index(const nnp_handle *h, const char *name, int32_t *index);
int nnp_rc(const nnp_handle *h, double *rc);
int nnp_n_input(const nnp_handle *h, int32_t type, int32_t *n_input);

/* Energies, forces and (optionally) symmetry functions of a batch.
 * Replaces NNP::compute(Structure&) (nnp.cpp:489-494) = NeighborList::build
 * (struc/neighbor.cpp:46-87) + NNP::compute_symm (nnp.cpp:350-392) +
 * NNP::compute_force (nnp.cpp:412-476), and NNP::compute_energy (nnp.cpp:329-338)
 * when NNP_VACUUM is set.
 *  energy[n_struct]   sum of atomic energies (plus vacuum energies with NNP_VACUUM)
 *  forces[3*N]        -dE/dr per atom
 *  symm_out[N*gstride] symmetry functions, row per atom, gstride = max n_input
 *                      (only with NNP_SYMM)
 * With NNP_DEVICE_PTRS all pointers (batch arrays and outputs) are device
 * pointers and nothing is copied; otherwise they are host pointers. */
int nnp_compute(nnp_handle *h, const nnp_batch *batch, double *energy, double *forces,
                double *symm_out, uint32_t flags);

/* Force call for molecular dynamics: nnp_compute plus the per-atom energies
 * and the virial of every structure, the outputs a LAMMPS-style pair style needs
 * (the reference's ML-ATOMNN pair style is not in its sources; its per-atom
 * energy is NNH::energy, nnh.cpp:207-210).  Any output may be NULL.
 *  energy[n_struct]      as nnp_compute
 *  forces[3*N]           as nnp_compute
 *  atom_energy[N]        network energy of each atom (plus its vacuum energy with NNP_VACUUM)
 *  virial[9*n_struct]    W = -dE/d(strain), W[9s+3a+b] = -sum over pairs of
 *                        (dE_i/dd)_a d_b for the displacements d = x_i - x_j - R q
 *                        (eV; the pressure tensor is W / volume)
 * flags: NNP_VACUUM, NNP_DEVICE_PTRS. */
int nnp_compute_md(nnp_handle *h, const nnp_batch *batch, double *energy, double *forces, double *atom_energy,
                   double *virial, uint32_t flags);

/* Force call of a LAMMPS-style pair style on one spatial domain (the
 * reference's ML-ATOMNN pair style, README.md:376-380, is not in its
 * sources): n_local owned atoms followed by n_ghost ghost atoms (periodic
 * images and neighbouring domains' atoms within rc of the domain, as the
 * caller's communication provides them), no cell.  Only local atoms are
 * centres: the energy is the sum of their atomic energies; ghosts enter
 * only as neighbours.  Forces are written for every atom, ghosts included
 * (-dE/dx_ghost, to be added to the owning atom by the caller's reverse
 * communication, as a pair style with newton on does).
 *  pos[3*(n_local+n_ghost)], type[n_local+n_ghost]   host arrays
 *  energy[1]                  sum of the local atoms' energies (+ vacuum with NNP_VACUUM)
 *  forces[3*(n_local+n_ghost)]
 *  atom_energy[n_local]       per-atom energies of the local atoms
 *  virial[9]                  W = -dE/d(strain) of the domain's pair terms
 *                             (sum over all atoms of x_i (x) F_i), as nnp_compute_md
 * Any output may be NULL.  flags: NNP_VACUUM. */
int nnp_compute_local_ghost(nnp_handle *h, int64_t n_local, int64_t n_ghost, const double *pos,
                            const int32_t *type, double *energy, double *forces, double *atom_energy,
                            double *virial, uint32_t flags);

/* Energy of every structure from precomputed symmetry functions; replaces
 * NNP::compute_energy (nnp.cpp:329-338) with NNH::energy (nnh.cpp:207-210):
 * sum over atoms of network(G) + vacuum energy.  symm is N*gstride (host). */
int nnp_compute_energy_symm(nnp_handle *h, int32_t n_struct, const int64_t *atom_off,
                            const int32_t *type, const double *symm, int32_t gstride,
                            double *energy);

/* Number of network parameters of one type / of all types (ANN::size, ml/nn.cpp:1000-1006). */
int nnp_nparams(const nnp_handle *h, int32_t type, int32_t *n);

/* All networks' parameters, types in index order, each in the reference packing
 * (biases by layer, then column-major weights): operator>> / operator<<
 * (ml/nn.cpp:881-915) as used by nnptefr (nnptefr.cpp:1171-1181). */
int nnp_get_params(const nnp_handle *h, double *params);
int nnp_set_params(nnp_handle *h, const double *params);

/* Energy(+force) loss and its gradient with respect to all network parameters.
 * The energy term is NNPTEFR::error_cost_o1's (nnptefr.cpp:1292-1380, batch
 * average nnptefr.cpp:996-1000), MSE unless nnp_set_loss picks another kind;
 * the force term has no reference counterpart in nnptefr (which trains on
 * energies only; its second derivatives are the reference's NN::D2ODZDI,
 * ml/nn.cpp:2047-2137, contracted with dG/dr):
 *   L = (1/B) sum_s [ 0.5*(norm_s*(E_s - e_ref_s))^2
 *                     + w_f * 0.5/(3 N_s) * sum_i |F_i - f_ref_i|^2 ]
 * E_s excludes vacuum energies (nnptefr subtracts them from the labels,
 * nnptefr.cpp:2958).  norm_mode: 0 IDENTITY, 1 LINEAR (1/N_s), 2 SQRT, 3 CBRT,
 * 4 LOG (nnptefr.cpp:614-620).  grad has nnp_nparams total entries in the
 * nnp_get_params order.  e_out / f_out (optional) receive the model's E, F.
 * The loss, its per-atom factors and the gradient are computed on the
 * device, and the gradient stays on the handle for nnp_opt_adam /
 * nnp_opt_step.  flags: 0 (host pointers) or NNP_DEVICE_PTRS: the batch
 * arrays, e_ref, f_ref, loss (one double), grad, e_out and f_out are then
 * device memory, grad may be NULL, and the call returns after one
 * synchronisation (the forward pass's error check) with the rest queued on
 * the handle's stream. */
int nnp_train_grad(nnp_handle *h, const nnp_batch *batch, const double *e_ref,
                   const double *f_ref, double w_f, int32_t norm_mode, double *loss,
                   double *grad, double *e_out, double *f_out, uint32_t flags);

/* Structure files into a CSR batch: extended XYZ, every frame of the file
 * (XYZ::read, format/xyz_struc.cpp:26-180: Properties=species:S:1:pos:R:3
 * [:forces:R:3], potential_energy=, Lattice="a1 a2 a3"; plain "name x y z"
 * lines when there is no Properties field; positions of a periodic frame
 * wrapped into its cell), or a VASP POSCAR/CONTCAR, one structure
 * (VASP::POSCAR::read, format/vasp_struc.cpp:41-190; as in the reference the scale
 * multiplies the lattice, not Cartesian positions).  METAL units (A, eV).
 * Element names are mapped to type indices by type_names[ntypes] (a
 * potential's names in index order, nnp_type_name; NNP::index); an unknown
 * name is NNP_ERR_TYPE.  Host only, no handle or GPU; errors in
 * nnp_last_error(NULL).  Call with atom_off = NULL to get the sizes
 * (*n_struct, *n_atoms); then with arrays of at least those sizes (in:
 * capacities, out: sizes): atom_off[n_struct+1], pos[3N], type[N],
 * cell[9 n_struct], pbc[n_struct] (1 when the frame has a lattice),
 * energy[n_struct] (0 when the file has none), forces[3N] (0 when none);
 * any of the last six may be NULL. */
#define NNP_FMT_XYZ 1
#define NNP_FMT_VASP 2
int nnp_read_structures(int32_t ntypes, const char *const *type_names, const char *path, int32_t format,
                        int32_t *n_struct, int64_t *n_atoms, int64_t *atom_off, double *pos, int32_t *type,
                        double *cell, int32_t *pbc, double *energy, double *forces);

/* Name of element `type` of the potential (NNP::nnh(type).type().name()). */
int nnp_type_name(const nnp_handle *h, int32_t type, const char **name);

/* Input statistics of the networks over a training set: NNPTEFR::train's
 * statistics of the symmetry functions per element (nnptefr.cpp:689-781),
 * computed on the device from the batch's symmetry functions (the
 * accumulation mode of nnp_set_accumulation applies).
 *  count[ntypes]                         atoms of each element
 *  stats[(t*NNP_NSTATS + s)*gstride + k] statistic s of input k of element t,
 *                                        gstride = max nnp_n_input (the rest is 0):
 *   NNP_STAT_MAX, NNP_STAT_MIN, NNP_STAT_HARMONIC (N / sum 1/G), NNP_STAT_MEAN,
 *   NNP_STAT_DEV (sqrt(sum (mean - G)^2 / (N - 1))), NNP_STAT_RMS (sqrt(sum G^2 / N)).
 * Host pointers. */
#define NNP_NSTATS 6
#define NNP_STAT_MAX 0
#define NNP_STAT_MIN 1
#define NNP_STAT_HARMONIC 2
#define NNP_STAT_MEAN 3
#define NNP_STAT_DEV 4
#define NNP_STAT_RMS 5
int nnp_input_stats(nnp_handle *h, const nnp_batch *batch, int64_t *count, double *stats);

/* Preconditioning of the network inputs from those statistics, as nnptefr
 * does before training (nnptefr.cpp:783-880): per element
 *   inpb = -(statistic of prebias) + inbias, inpw = (1 / statistic of prescale) * inscale,
 * outb = 0, outw = 1.  prebias: PreBias (nnptefr.hpp:97-107) IDENTITY 0 (inpb = 0),
 * MEAN 1, HAR 2, RMS 3, MID 4 ((max+min)/2), MIN 5; prescale: PreScale
 * (nnptefr.hpp:69-77) IDENTITY 0 (inpw = 1), DEV 1, MINMAX 2 (max - min), MAX 3;
 * a zero (DEV, MINMAX) or non-positive (MAX) statistic gives scale 1.
 * The reference's NONE values (6, 4) are rejected like the reference rejects
 * them ("Invalid input bias." / "Invalid input scaling.").  The handle's
 * networks are updated in place; nnp_write writes them. */
#define NNP_PREBIAS_IDENTITY 0
#define NNP_PREBIAS_MEAN 1
#define NNP_PREBIAS_HAR 2
#define NNP_PREBIAS_RMS 3
#define NNP_PREBIAS_MID 4
#define NNP_PREBIAS_MIN 5
#define NNP_PRESCALE_IDENTITY 0
#define NNP_PRESCALE_DEV 1
#define NNP_PRESCALE_MINMAX 2
#define NNP_PRESCALE_MAX 3
int nnp_precondition(nnp_handle *h, const nnp_batch *batch, int32_t prebias, int32_t prescale, double inbias,
                     double inscale);

/* Taylor expansion of a training set (NNPTEFR's force perturbation,
 * nnptefr.cpp:2733-2830), on the current CUDA device, no handle: each
 * structure whose mean force norm exceeds 1e-12 is followed by nadd copies
 * in which every atom j moves by dr_j = vr (sin t cos p, sin t sin p, cos t)
 * (cos t, p / pi uniform in (-1, 1)) with vr drawn from distribution dist of
 * width rdelta -- rng::dist::Name (math/random.hpp:32-42): 1 UNIFORM(0, w),
 * 2 LAPLACE(0, w), 3 NORMAL(0, w), 5 SECH(0, w), 6 LOGISTIC(0, w), 7 COSINE(0, w)
 * -- and whose energy is E - sum_j dr_j . F_j.  The random numbers are a
 * counter-based hash of (seed, output structure, atom): the same inputs and
 * seed give the same copies (the reference's std::mt19937 stream is not
 * reproduced).  Host arrays.  Outputs hold up to n_struct * (1 + nadd)
 * structures: out_atom_off[n_out+1], out_pos[3*atoms], out_type[atoms],
 * out_energy[n_out], out_src[n_out] (the source structure of each, whose
 * cell the caller reuses), *n_out.  Errors: nnp_last_error(NULL). */
int nnp_taylor_expand(int32_t n_struct, const int64_t *atom_off, const double *pos, const int32_t *type,
                      const double *energy, const double *forces, int32_t nadd, int32_t dist, double rdelta,
                      uint64_t seed, int64_t *out_atom_off, double *out_pos, int32_t *out_type, double *out_energy,
                      int32_t *out_src, int32_t *n_out);

/* Energy-loss kind of nnp_train_grad, opt::Loss (opt/loss.hpp:18-24) as
 * NNPTEFR::error_cost_o1 applies it to dU = norm_s (E_s - e_ref_s)
 * (nnptefr.cpp:1340-1376): MSE 0.5 dU^2 (the default), MAE |dU|,
 * HUBER delta^2 (sqrt(1 + (dU/delta)^2) - 1),
 * ASINH delta^2 (1 - sqrt(1 + a^2) + a asinh(a)), a = dU/delta.
 * The force term stays the MSE of nnp_train_grad.  delta (> 0) is used by
 * HUBER and ASINH only. */
#define NNP_LOSS_MSE 1
#define NNP_LOSS_MAE 2
#define NNP_LOSS_HUBER 3
#define NNP_LOSS_ASINH 4
int nnp_set_loss(nnp_handle *h, int32_t kind, double delta);

/* One ADAM step on the device (opt::algo::ADAM::step, opt/algo.cpp:280-296,
 * beta1 0.9, beta2 0.999) with the gradient of the last nnp_train_grad,
 * which stays on the device: m = b1 m + (1-b1) g, v = b2 v + (1-b2) g^2,
 * p -= gamma m / (1 - b1^t) / (sqrt(v / (1 - b2^t)) + eps).  The running
 * averages and an FP64 master copy of the parameters live on the handle
 * (zeroed at the first step, as ADAM::resize); the networks the next call
 * uses are updated on the device, and the host model (nnp_get_params,
 * nnp_write) is updated with them.  The learning rate gamma is the caller's
 * (the reference's decay schedules set it per step).  nnp_opt_reset
 * restarts the averages.  nnptefr's binary restart file is not read or written. */
int nnp_opt_adam(nnp_handle *h, double gamma, double eps);
int nnp_opt_reset(nnp_handle *h);

/* The learning-rate schedules of opt::Decay::step (opt/decay.cpp:58-82,
 * names decay.hpp:28-36): the rate of the next step from the current one,
 * at iteration step.  Host only; errors in nnp_last_error(NULL). */
#define NNP_DECAY_CONST 1   /* gamma                                           */
#define NNP_DECAY_EXP 2     /* gamma (1 - alpha)                               */
#define NNP_DECAY_GAUSS 3   /* gamma (1 - 2 alpha step)                        */
#define NNP_DECAY_SQRT 4    /* gamma (1 - alpha / 2 / (1 + alpha step))       */
#define NNP_DECAY_INV 5     /* gamma (1 - alpha / (1 + alpha step))           */
#define NNP_DECAY_STEP 6    /* gamma alpha when step > 0 is a multiple of period */
int nnp_decay_step(int32_t kind, double alpha, int32_t period, double gamma, int32_t step, double *out);

/* One optimiser step of nnptefr's loop (nnptefr.cpp:1032-1057) on the device:
 * *gamma = decay(*gamma, step), the ADAM step of nnp_opt_adam with it, then
 * weight decay of the weights (not the biases) at their values before the
 * step, p -= gamma eta r(p): regularization (nnptefr.hpp:183-191) LASSO
 * sgn(p), RIDGE p, HUBER p / sqrt(1 + p^2), ASINH asinh(p), or NONE.
 * *gamma receives the rate used. */
#define NNP_REG_LASSO 0
#define NNP_REG_RIDGE 1
#define NNP_REG_HUBER 2
#define NNP_REG_ASINH 3
#define NNP_REG_NONE 4
int nnp_opt_step(nnp_handle *h, double *gamma, int32_t step, int32_t decay_kind, double alpha, int32_t period,
                 int32_t reg_kind, double eta, double eps);

/* Allocation-free energies from device-resident symmetry functions (no
 * counterpart in the reference, whose NNP::compute_energy (nnp.cpp:329-338)
 * it otherwise follows).  For callers that must not allocate device memory
 * during the call -- cudaMalloc/cudaFree synchronise the device and can fail
 * once a serving process has reserved its memory -- this call allocates
 * nothing: its only scratch (one float per atom) is a fixed array inside the
 * library, so a call takes at most NNP_NOALLOC_MAX_ATOMS atoms (larger
 * batches return NNP_ERR_CAPACITY before anything is launched).
 *  d_atom_off[n_struct+1], d_type[n_atoms], d_symm[n_atoms*gstride] (FP32 rows,
 *  gstride >= the largest nnp_n_input), d_energy[n_struct] (FP64 out) are
 *  device pointers on the handle's device, which must be current; n_atoms
 *  must equal d_atom_off[n_struct] (a structure whose offsets fall outside
 *  [0, n_atoms] gets a NaN energy).  flags: 0 or NNP_VACUUM.
 * The networks are the FP32 ones: a handle set to NNP_PREC_BF16 or
 * NNP_PREC_BF16X3 gets NNP_ERR_UNSUPPORTED (set NNP_PREC_FP32 first).
 * The kernels are queued on the handle's stream and the call returns without
 * waiting for them.  An atom type outside [0, ntypes) gives a NaN energy for
 * its structure.  The first call on a handle looks up the scratch array's
 * device address (which may load the library's device code) and keeps it
 * with the handle; make that first call before any stream capture.  The
 * scratch array is one per device, shared by all handles: calls that can
 * overlap in time (other streams, other host threads) race on it and must be
 * ordered by the caller. */
#define NNP_NOALLOC_MAX_ATOMS (1 << 20)
int nnp_energy_symm_noalloc(nnp_handle *h, int32_t n_struct, int64_t n_atoms, const int64_t *d_atom_off,
                            const int32_t *d_type, const float *d_symm, int32_t gstride, uint32_t flags,
                            double *d_energy);

/* Stage timers, the device-side counterpart of the reference's phase clocks
 * ("time - symm/energy/force", nnptefr.cpp:2863-2885, 3547-3592).  When enabled,
 * nnp_compute records CUDA events between its stages; nnp_stage_times then
 * returns the last call's durations in ms: [0] neighbour list, [1] symmetry
 * functions, [2] networks, [3] forces, [4] energies. */
int nnp_set_timing(nnp_handle *h, int32_t enable);
int nnp_stage_times(const nnp_handle *h, float *ms, int32_t n);

/* Neighbour counts of the last nnp_compute, split by neighbour type:
 * counts[i*ntypes + t] is the number of type-t neighbours of atom i (host
 * array of N*ntypes).  The pair and triplet counts per atom follow from these
 * (NeighborList::size, struc/neighbor.hpp:35). */
int nnp_neighbor_counts(nnp_handle *h, int32_t *counts);

/* Kernels this handle has launched since it was created. */
int nnp_launch_count(const nnp_handle *h, int64_t *n);

/* Message of the last error on this handle (or, when h is NULL, of the last
 * failed create or handle-free call such as nnp_taylor_expand). */
const char *nnp_last_error(const nnp_handle *h);

/* Library version string. */
const char *nnp_version(void);

#ifdef __cplusplus
}
#endif
#endif
