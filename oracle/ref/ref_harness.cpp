// ref_harness.cpp -- C-callable wrapper around the reference's own NNP code
// (NNP::read, NNP::init, NeighborList::build, NNP::compute_symm,
// NNP::compute_force, NNP::compute_energy), compiled from the reference
// sources by oracle/ref/Makefile.  TEST INFRASTRUCTURE ONLY: it lets the
// tests and the CPU baseline call the reference itself through ctypes.
#include <cstring>
#include <exception>
#include <string>

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
        Atom atom;
        atom.name() = true;
        atom.type() = true;
        atom.posn() = true;
        atom.force() = true;
        atom.symm() = true;
        Structure struc(n, atom);
        Eigen::Matrix3d R = Eigen::Matrix3d::Zero();
        if (pbc)
            for (int c = 0; c < 3; ++c)
                for (int d = 0; d < 3; ++d) R(d, c) = cell[3 * c + d];
        if (pbc) struc.init(R);
        for (int i = 0; i < n; ++i) {
            struc.type(i) = type[i];
            struc.name(i) = nnp.nnh(type[i]).type().name();
            for (int d = 0; d < 3; ++d) struc.posn(i)[d] = pos[3 * i + d];
        }
        nnp.init(struc);
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

}  // extern "C"
