// nnp_internal.h -- host-side model of a potential and the text-format
// readers/writers.  The device-side layout lives in nnp_device.cuh.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "nnp_device.cuh"

namespace nnp {

struct HostBasisR { int cut = 0; double rc = 0; int form = 0; std::vector<double> rs, eta; };
struct HostBasisA { int cut = 0; double rc = 0; int form = 0; std::vector<double> eta, zeta; std::vector<int> lambda; };
struct HostNet {
    std::vector<int> nodes;               // nodes[0] = inputs, ..., nodes.back() = outputs
    int neuron = 0;
    double c = 1.0;
    std::vector<double> inpw, inpb, outw, outb;
    std::vector<std::vector<double>> b;   // b[l][n]
    std::vector<std::vector<double>> w;   // w[l][n*nin + m] row-major (n_out x n_in)
    int nparams() const;
};
struct HostType {
    std::string name;
    double energy = 0, mass = 0, charge = 0, radius = 0, z = 0, alpha = 0, ie = 0, rcov = 0, rvdw = 0, amp = 0;
};
struct HostPot {
    std::vector<HostType> types;
    double rc = 0;
    std::vector<std::vector<HostBasisR>> br;   // [II][J]
    std::vector<std::vector<HostBasisA>> ba;   // [II][tt]
    std::vector<HostNet> nets;                  // [II]
    int ntypes() const { return (int)types.size(); }
    int n_input_r(int II) const;
    int n_input(int II) const;
};

int tt_index(int i, int j);
// Parsers/writers of the reference text formats; they return an empty string
// on success or an error message.
std::string read_potential(const std::string &text, HostPot &pot);
std::string write_potential(const HostPot &pot);
std::string read_basis_file(const std::string &text, HostPot &pot, int II);
std::string read_network(const std::string &text, HostNet &net);

// One structure read from a structure file (nnp_read_structures).
struct ReadStruct {
    std::vector<std::string> names;   // element of each atom
    std::vector<double> pos;          // 3 per atom, A
    std::vector<double> forces;       // 3 per atom, eV/A (zero when the file has none)
    double cell[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};   // cell[3n+d]: component d of lattice vector n
    double energy = 0;                // potential energy, eV
    bool pbc = false, has_forces = false;
};
std::string read_xyz_frames(const std::string &text, std::vector<ReadStruct> &out);
std::string read_vasp(const std::string &text, std::vector<ReadStruct> &out);

// A network's floats in wpar, starting at DevType::woff:
//   inpw[nin], inpb[nin], outw[nout], outb[nout],
//   then for each layer l: bias[no] and the weights transposed with a padded
//   row, W^T[m * wt_stride(no) + n] = W[n][m]  (m < ni, n < no).
int64_t net_floats(const HostNet &net);

}  // namespace nnp
