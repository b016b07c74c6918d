// ref_harness.cpp -- C-callable wrapper around the reference's own NNP code
// (NNP::read, NNP::init, NeighborList::build, NNP::compute_symm,
// NNP::compute_force, NNP::compute_energy, and the training-side NN::ANN::fpbp,
// NN::Cost::grad and NN::D2ODZDI::grad), compiled from the reference sources
// by oracle/ref/Makefile.  TEST INFRASTRUCTURE ONLY: it lets the tests, the
// fixture generator and the CPU baseline call the reference itself through
// ctypes.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "format/vasp_struc.hpp"
#include "format/xyz_struc.hpp"
#include "ml/nn.hpp"
#include "opt/decay.hpp"
#include "opt/iter.hpp"
#include "nnp/nnp.hpp"
#include "struc/neighbor.hpp"
#include "struc/structure.hpp"

namespace {
void put(char *err, int len, const std::string &s)
{
    if (err && len > 0) {
        std::strncpy(err, s.c_str(), (size_t)len - 1);
        err[len - 1] = '\0';
    }
}

// A Structure holding n atoms of the NNP's types at pos[3n], lattice vectors
// cell[3c+d] (component d of vector c) when pbc, sized for the NNP (NNP::init).
void make_structure(NNP &nnp, int n, const double *pos, const int *type, const double *cell, int pbc,
                    Structure &struc)
{
    Atom atom;
    atom.name() = true;
    atom.type() = true;
    atom.posn() = true;
    atom.force() = true;
    atom.symm() = true;
    struc = Structure(n, atom);
    if (pbc) {
        Eigen::Matrix3d R = Eigen::Matrix3d::Zero();
        for (int c = 0; c < 3; ++c)
            for (int d = 0; d < 3; ++d) R(d, c) = cell[3 * c + d];
        struc.init(R);
    }
    for (int i = 0; i < n; ++i) {
        struc.type(i) = type[i];
        struc.name(i) = nnp.nnh(type[i]).type().name();
        for (int d = 0; d < 3; ++d) struc.posn(i)[d] = pos[3 * i + d];
    }
    nnp.init(struc);
}

// Symmetry functions of one structure: NeighborList::build + NNP::compute_symm.
void symm_of(NNP &nnp, int n, const double *pos, const int *type, const double *cell, int pbc,
             std::vector<Eigen::VectorXd> &G)
{
    Structure struc;
    make_structure(nnp, n, pos, type, cell, pbc, struc);
    NeighborList nlist(nnp.rc());
    nlist.build(struc);
    nnp.compute_symm(struc, nlist);
    G.resize(n);
    for (int i = 0; i < n; ++i) G[i] = struc.symm(i);
}

// nnptefr's per-structure normalisation (nnptefr.cpp:614-620).
double norm_factor(int mode, double nat)
{
    switch (mode) {
    case 0: return 1.0;
    case 1: return 1.0 / nat;
    case 2: return 1.0 / std::sqrt(nat);
    case 3: return 1.0 / std::cbrt(nat);
    case 4: return 1.0 / (std::log(nat) + 1.0);
    default: throw std::invalid_argument("Invalid normalization method.");
    }
}
}  // namespace

extern "C" {

void *ref_nnp_read(const char *path, char *err, int errlen)
{
    try {
        NNP *p = new NNP();
        NNP::read(path, *p);
        return p;
    } catch (std::exception &e) {
        put(err, errlen, e.what());
    }
    return nullptr;
}

void ref_nnp_free(void *h) { delete static_cast<NNP *>(h); }

int ref_nnp_ntypes(void *h) { return static_cast<NNP *>(h)->ntypes(); }

double ref_nnp_rc(void *h) { return static_cast<NNP *>(h)->rc(); }

int ref_nnp_ninput(void *h, int type) { return static_cast<NNP *>(h)->nnh(type).nInput(); }

// Parameters of one type's network (ANN::size, ml/nn.cpp:1000-1006).
int ref_nnp_nparams(void *h, int type) { return static_cast<NNP *>(h)->nnh(type).nn().size(); }

// One structure: n atoms, positions pos[3n], NNP type indices type[n],
// lattice vectors cell[3c+d] (component d of vector c), periodic if pbc
// (otherwise a zero cell, for which NeighborList::build searches no images).
// Outputs: energy = NNP::compute_force's pe (no vacuum energies),
// forces[3n], symm[n*gstride] (optional), energy_vac = NNP::compute_energy
// (optional, network energies + vacuum energies).
int ref_nnp_compute(void *h, int n, const double *pos, const int *type, const double *cell, int pbc, int gstride,
                    double *energy, double *forces, double *symm, double *energy_vac, char *err, int errlen)
{
    try {
        NNP &nnp = *static_cast<NNP *>(h);
        Structure struc;
        make_structure(nnp, n, pos, type, cell, pbc, struc);
        NeighborList nlist(nnp.rc());
        nlist.build(struc);
        nnp.compute_symm(struc, nlist);
        const double pe = nnp.compute_force(struc, nlist);
        if (energy) *energy = pe;
        if (forces)
            for (int i = 0; i < n; ++i)
                for (int d = 0; d < 3; ++d) forces[3 * i + d] = struc.force(i)[d];
        if (symm)
            for (int i = 0; i < n; ++i)
                for (int g = 0; g < gstride; ++g) symm[(size_t)i * gstride + g] = g < struc.symm(i).size() ? struc.symm(i)[g] : 0.0;
        if (energy_vac) *energy_vac = nnp.compute_energy(struc);
        return 0;
    } catch (std::exception &e) {
        put(err, errlen, e.what());
    }
    return -1;
}

// Energy-loss gradient of a batch with the reference's own training code:
// per structure NeighborList::build + NNP::compute_symm, then, per atom,
// NN::ANN::fpbp and NN::Cost::grad with dc/do = 1 (ml/nn.cpp:1402-1420,
// 1747-1805), accumulated per element and scaled by the loss factor exactly as
// NNPTEFR::error_cost_o1 does (nnptefr.cpp:1331-1380), then averaged over the
// batch (nnptefr.cpp:996-1000).  loss_kind follows opt::Loss (1 MSE, 2 MAE,
// 3 HUBER, 4 ASINH; opt/loss.hpp:18-24) with width delta; norm_mode follows
// nnptefr's Norm (0 IDENTITY, 1 LINEAR, 2 SQRT, 3 CBRT, 4 LOG).
// grad receives the per-element gradients, types in index order, each in the
// reference packing (biases by layer, then column-major weights).
// Outputs: *loss (error_[0] averaged), *rmse (error_[2] averaged, then sqrt),
// energy[nstruct] (the network energies pe).
int ref_energy_loss_grad(void *h, int nstruct, const int64_t *atom_off, const double *pos, const int *type,
                         const double *cell, int pbc, const double *e_ref, int norm_mode, int loss_kind,
                         double delta, double *grad, double *loss, double *rmse, double *energy, char *err,
                         int errlen)
{
    try {
        NNP &nnp = *static_cast<NNP *>(h);
        const int T = nnp.ntypes();
        std::vector<NN::Cost> cost(T);
        std::vector<Eigen::VectorXd> gElement(T), gStruc(T);
        for (int t = 0; t < T; ++t) {
            cost[t].resize(nnp.nnh(t).nn());
            gElement[t] = Eigen::VectorXd::Zero(nnp.nnh(t).nn().size());
            gStruc[t] = Eigen::VectorXd::Zero(nnp.nnh(t).nn().size());
        }
        const double deltai = 1.0 / delta, delta2 = delta * delta;
        double err0 = 0, err2 = 0;
        const Eigen::VectorXd dcdo = Eigen::VectorXd::Constant(1, 1);
        std::vector<Eigen::VectorXd> G;
        for (int s = 0; s < nstruct; ++s) {
            const int64_t a0 = atom_off[s];
            const int n = (int)(atom_off[s + 1] - a0);
            symm_of(nnp, n, pos + 3 * a0, type + a0, cell + 9 * s, pbc, G);
            for (int t = 0; t < T; ++t) gStruc[t].setZero();
            double pe = 0;
            for (int i = 0; i < n; ++i) {
                const int t = type[a0 + i];
                nnp.nnh(t).nn().fpbp(G[i]);
                pe += nnp.nnh(t).nn().out()[0];
                gStruc[t].noalias() += cost[t].grad(nnp.nnh(t).nn(), dcdo);
            }
            if (energy) energy[s] = pe;
            const double nat = n;
            const double nrm = norm_factor(norm_mode, nat);
            const double dE = pe - e_ref[s];
            const double dU = dE * nrm;
            double gfac = nrm;
            switch (loss_kind) {
            case 1: err0 += 0.5 * dU * dU; gfac *= dU; break;
            case 2: err0 += std::fabs(dU); gfac *= (dU > 0) - (dU < 0); break;
            case 3: {
                const double arg = dU * deltai, sq = std::sqrt(1.0 + arg * arg);
                err0 += delta2 * (sq - 1.0);
                gfac *= dU / sq;
            } break;
            case 4: {
                const double arg = dU * deltai, sq = std::sqrt(1.0 + arg * arg), lg = std::log(arg + sq);
                err0 += delta2 * (1.0 - sq + arg * lg);
                gfac *= lg * delta;
            } break;
            default: throw std::invalid_argument("Invalid loss.");
            }
            err2 += (dE * dE) / (nat * nat);
            for (int t = 0; t < T; ++t) gElement[t].noalias() += gStruc[t] * gfac;
        }
        const double bi = 1.0 / nstruct;
        size_t k = 0;
        for (int t = 0; t < T; ++t)
            for (int p = 0; p < gElement[t].size(); ++p) grad[k++] = gElement[t][p] * bi;
        if (loss) *loss = err0 * bi;
        if (rmse) *rmse = std::sqrt(err2 * bi);
        return 0;
    } catch (std::exception &e) {
        put(err, errlen, e.what());
    }
    return -1;
}

// Weight gradient of sum_i dE_i/dG_i . C_i for one structure, where
// C_i = sum_k dG_i/dx_k . v_k is the change of atom i's symmetry functions
// along the displacement field v (v[3n]).  The second derivatives come from
// the reference's NN::D2ODZDI::grad (ml/nn.cpp:2047-2137, after
// NN::ANN::fpbp2, nn.cpp:1426-1444): grad_p += sum_k d2o/dp dI_k * C_ik.
// C_i is taken by central differences of the reference's own
// NNP::compute_symm at x + fd_h v and x - fd_h v.  D2ODZDI differentiates
// with respect to the raw input and omits the input scale inpw in its
// first-layer weight term, so it is exact only for networks with inpw = 1
// (the setting of the reference's own test, ml/test_nn_grad.cpp:420-423);
// callers pass such a potential.  With v = the force-loss adjoint
// w_f (F - F_ref) / (3 N B), -grad is the force term of the loss gradient.
// grad has the per-element packing of ref_energy_loss_grad and is ADDED to;
// ctan (optional, n rows of the largest nInput) receives the C_i.
int ref_force_term_grad(void *h, int n, const double *pos, const int *type, const double *cell, int pbc,
                        const double *v, double fd_h, double *grad, double *ctan, char *err, int errlen)
{
    try {
        NNP &nnp = *static_cast<NNP *>(h);
        const int T = nnp.ntypes();
        std::vector<double> xp(3 * (size_t)n), xm(3 * (size_t)n);
        for (int k = 0; k < 3 * n; ++k) {
            xp[k] = pos[k] + fd_h * v[k];
            xm[k] = pos[k] - fd_h * v[k];
        }
        std::vector<Eigen::VectorXd> G0, Gp, Gm;
        symm_of(nnp, n, pos, type, cell, pbc, G0);
        symm_of(nnp, n, xp.data(), type, cell, pbc, Gp);
        symm_of(nnp, n, xm.data(), type, cell, pbc, Gm);
        std::vector<int> off(T + 1, 0);
        for (int t = 0; t < T; ++t) off[t + 1] = off[t] + nnp.nnh(t).nn().size();
        std::vector<NN::D2ODZDI> d2(T);
        int gstride = 0;
        for (int t = 0; t < T; ++t) {
            d2[t].resize(nnp.nnh(t).nn());
            gstride = std::max(gstride, nnp.nnh(t).nInput());
        }
        for (int i = 0; i < n; ++i) {
            const int t = type[i];
            NN::ANN &nn = nnp.nnh(t).nn();
            const Eigen::VectorXd C = (Gp[i] - Gm[i]) / (2.0 * fd_h);
            if (ctan)
                for (int q = 0; q < C.size(); ++q) ctan[(size_t)i * gstride + q] = C[q];
            nn.fpbp2(G0[i]);
            d2[t].resize(nn);  // D2ODZDI::grad adds into d2odzdi_, which only resize() zeroes
            d2[t].grad(nn);
            for (int p = 0; p < nn.size(); ++p) {
                const Eigen::MatrixXd &M = d2[t].d2odpdi()[p];
                double s = 0;
                for (int q = 0; q < C.size(); ++q) s += M(0, q) * C[q];
                grad[off[t] + p] += s;
            }
        }
        return 0;
    } catch (std::exception &e) {
        put(err, errlen, e.what());
    }
    return -1;
}

// One structure file through the reference's own reader: format 1 extended
// XYZ (XYZ::read, first frame), 2 VASP POSCAR (VASP::read).  Writes the atom
// count, positions[3n], forces[3n], pe, the lattice vectors cell[3c+d]
// (zero without a cell) and the element names, one per line, into names.
int ref_read_structure(const char *path, int format, int cap, int *n, double *pos, double *forces, double *pe,
                       double *cell, char *names, int names_len, char *err, int errlen)
{
    try {
        Atom atom;
        atom.name() = true;
        atom.type() = true;
        atom.posn() = true;
        atom.force() = true;
        Structure struc;
        if (format == 1) XYZ::read(path, atom, struc);
        else VASP::POSCAR::read(path, atom, struc);
        *n = struc.nAtoms();
        if (struc.nAtoms() > cap) throw std::runtime_error("too many atoms");
        for (int i = 0; i < struc.nAtoms(); ++i)
            for (int d = 0; d < 3; ++d) {
                pos[3 * i + d] = struc.posn(i)[d];
                forces[3 * i + d] = format == 1 ? struc.force(i)[d] : 0.0;
            }
        *pe = struc.pe();
        const Eigen::Matrix3d R = struc.R();
        for (int c = 0; c < 3; ++c)
            for (int d = 0; d < 3; ++d) cell[3 * c + d] = R(d, c);
        std::string all;
        for (int i = 0; i < struc.nAtoms(); ++i) all += struc.name(i) + "\n";
        put(names, names_len, all);
        return 0;
    } catch (std::exception &e) {
        put(err, errlen, e.what());
    }
    return -1;
}

// opt::Decay::step (opt/decay.cpp:58-82) of decay kind `kind` (opt::Decay::Name)
// with alpha and period at iteration step.
double ref_decay_step(int kind, double alpha, int period, double gamma, int step)
{
    opt::Decay d(static_cast<opt::Decay::Name::Type>(kind), alpha);
    d.period() = period;
    opt::Iterator it;
    it.step() = step;
    return d.step(gamma, it);
}

}  // extern "C"
