/*
 * oracle.h -- FP64 CPU restatement of the reference NNP hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it.  The product (ace_b200/libnnp_b200.so) never links or calls it.
 *
 * Every function restates, in plain C, the arithmetic of the reference
 * (markdellostritto/ace, C++/Eigen, FP64) in the same operation order, so
 * that on the same inputs it reproduces the reference's numbers to the last
 * few ulps.  Citations are file:line inside the reference's src/ tree.
 *
 * Pinning: the restatement is checked against outputs of the reference's own
 * sources (compiled in place by oracle/ref/Makefile into oracle/_ref/) through
 * the golden fixtures under tests/golden/.
 */
#ifndef NNP_ORACLE_H
#define NNP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Cutoff::Name (nnp/cutoff.hpp:23-29) */
enum { ORC_CUT_NONE = 0, ORC_CUT_STEP, ORC_CUT_COS, ORC_CUT_TANH, ORC_CUT_POLY3 };
/* BasisR::Name (nnp/basis_radial.hpp:27-35) */
enum { ORC_R_NONE = 0, ORC_R_GAUSSIAN, ORC_R_SECH, ORC_R_LOGISTIC, ORC_R_TANH, ORC_R_LOGCOSH, ORC_R_LOGCOSH2 };
/* BasisA::Name (nnp/basis_angular.hpp:27-35) */
enum { ORC_A_NONE = 0, ORC_A_GAUSS, ORC_A_GAUSS2, ORC_A_SECH, ORC_A_STUDENT3, ORC_A_STUDENT4, ORC_A_STUDENT5 };
/* NN::Neuron (ml/nn.hpp:84-112) */
enum {
    ORC_NEU_NONE = 0, ORC_NEU_LINEAR, ORC_NEU_SIGMOID, ORC_NEU_TANH, ORC_NEU_ISRU, ORC_NEU_ARCTAN,
    ORC_NEU_RELU, ORC_NEU_ELU, ORC_NEU_TANHRE, ORC_NEU_SQRE, ORC_NEU_SWISH, ORC_NEU_GELU,
    ORC_NEU_MISH, ORC_NEU_PFLU, ORC_NEU_LOGISH, ORC_NEU_SOFTPLUS, ORC_NEU_SQPLUS, ORC_NEU_ATISH,
    ORC_NEU_IERF, ORC_NEU_TEST
};
#define ORC_MAX_LAYERS 8

/*
 * A whole potential, flattened.  T = ntypes, TT = T*(T+1)/2.
 * Radial block (II,J) lives at index II*T+J; angular block (II,jk) at
 * II*TT+jk where jk is the TensorTri rank-2 index (nnp/tensortri.hpp:196-200).
 * Basis parameters of block b start at r_off[b] / a_off[b].
 * Network of type II: nn_nodes[II*ORC_MAX_LAYERS + l] (l=0 is the input
 * size, l=1..nlayer the layer sizes); its doubles start at nn_off[II] and
 * hold inpw[nin], inpb[nin], outw[nout], outb[nout], then the parameter
 * vector in the reference packing (ml/nn.cpp:881-915): all biases by layer,
 * then every weight matrix column-major (n_out x n_in).
 */
typedef struct {
    int32_t ntypes;
    double rc;
    const int32_t *r_cut; const double *r_rc; const int32_t *r_form; const int32_t *r_n; const int32_t *r_off;
    const double *r_rs; const double *r_eta;
    const int32_t *a_cut; const double *a_rc; const int32_t *a_form; const int32_t *a_n; const int32_t *a_off;
    const double *a_eta; const double *a_zeta; const int32_t *a_lambda;
    const int32_t *n_input; const int32_t *n_input_r;
    const int32_t *offset_r; const int32_t *offset_a;
    const int32_t *nn_nlayer; const int32_t *nn_nodes; const int32_t *nn_neuron; const double *nn_c;
    const int64_t *nn_off; const double *nn_par;
    const double *energy; /* per-type vacuum energy, NNH::Type::energy */
} orc_pot;

/* ---- scalar building blocks (exported for unit tests) ---- */
double orc_fmexp(double x);                 /* math/special.cpp:249-284 */
double orc_coscut(double x);                /* math/special.cpp:21-27 */
double orc_sincut(double x);                /* math/special.cpp:35-41 */
double orc_cutf(int cut, double rc, double dr);  /* nnp/cutoff.cpp:62-86 */
double orc_cutg(int cut, double rc, double dr);  /* nnp/cutoff.cpp:88-114 */

/* ---- neighbour list, NeighborList::build (struc/neighbor.cpp:46-87) ----
 * pos: natoms x 3 (row per atom); cell: 9 doubles, cell[3*n+d] = component d
 * of lattice vector n (the columns of Cell::R).  pbc==0 means R=0 (no images).
 * Writes at most cap entries per atom into idx[i*cap+..] and img[(i*cap+..)*3+d];
 * counts[i] receives the full count even when it exceeds cap.
 * Returns 0, or -1 when some atom overflowed cap. */
int orc_nlist(double rc, int natoms, const double *pos, const double *cell, int pbc,
              int cap, int32_t *counts, int32_t *idx, double *img);

/* ---- NNP::compute_symm (nnp/nnp.cpp:350-392), brute-force neighbour list ----
 * symm: natoms x gstride (row per atom, nInput of the atom's type used). */
int orc_compute_symm(const orc_pot *pot, int natoms, const double *pos, const int32_t *type,
                     const double *cell, int pbc, int gstride, double *symm);

/* ---- NNP::compute_energy (nnp/nnp.cpp:329-338): sum of nn(G)+E_vac ---- */
double orc_compute_energy(const orc_pot *pot, int natoms, const int32_t *type, int gstride,
                          const double *symm);

/* ---- NNP::compute_force (nnp/nnp.cpp:412-476): needs symm from compute_symm;
 * returns E without vacuum energies; force: natoms x 3.  If dedg != NULL the
 * per-atom dE/dG rows (natoms x gstride) are written too. */
double orc_compute_force(const orc_pot *pot, int natoms, const double *pos, const int32_t *type,
                         const double *cell, int pbc, int gstride, const double *symm,
                         double *force, double *dedg);

/* ---- NNP::compute (nnp/nnp.cpp:489-494) = build + symm + force ---- */
double orc_compute(const orc_pot *pot, int natoms, const double *pos, const int32_t *type,
                   const double *cell, int pbc, int gstride, double *symm, double *force);

/* ---- single network ops on type II ---- */
/* ANN::fpbp (ml/nn.cpp:1402-1420) then DODZ::grad (ml/nn.cpp:1836-1859):
 * returns out[0]; dodi (nin) may be NULL. */
double orc_ann_fpbp(const orc_pot *pot, int II, const double *inp, double *dodi);
/* ANN::fpbp then Cost::grad with dcdo = 1 (ml/nn.cpp:1747-1805): grad has
 * nparams(II) entries in the reference packing. Returns out[0]. */
double orc_cost_grad(const orc_pot *pot, int II, const double *inp, double *grad);
int orc_nparams(const orc_pot *pot, int II);

/* ---- energy loss + gradient over a batch (nnptefr.cpp:1292-1380, the
 * batch average of nnptefr.cpp:996-1000).  Structures are CSR by atom_off.
 * norm_mode: 0 IDENTITY, 1 LINEAR (1/N), 2 SQRT, 3 CBRT, 4 LOG (nnptefr.cpp:614-620).
 * loss_kind: opt::Loss (opt/loss.hpp:18-24) 1 MSE, 2 MAE, 3 HUBER, 4 ASINH,
 * width delta (HUBER, ASINH).
 * grad: sum over types of nparams(type), types in index order.  Returns loss. */
double orc_energy_loss_grad(const orc_pot *pot, int nstruct, const int64_t *atom_off,
                            const int32_t *type, int gstride, const double *symm,
                            const double *e_ref, int norm_mode, int loss_kind, double delta,
                            double *grad);

/* ---- energy + force loss and its weight gradient (the nnptefr energy term
 * plus a force-weighted MSE term), for MSE:
 *   L = (1/B) sum_s [ 0.5*(norm_s*(E_s-E_ref_s))^2
 *                     + w_f * 0.5/(3 N_s) * sum_i |F_i - F_ref_i|^2 ]
 * and the energy term of orc_energy_loss_grad's loss_kind otherwise.
 * E_s excludes vacuum energies (compute_force semantics, as nnptefr subtracts
 * them from the labels).  Positions/cells/types are per structure (CSR).
 * grad may be NULL.  Returns L; eout (nstruct) and fout (N x 3) optional. */
double orc_ef_loss_grad(const orc_pot *pot, int nstruct, const int64_t *atom_off,
                        const double *pos, const int32_t *type, const double *cell, int pbc,
                        const double *e_ref, const double *f_ref, double w_f, int norm_mode,
                        int loss_kind, double delta, double *grad, double *eout, double *fout);

#ifdef __cplusplus
}
#endif
#endif
