// nnp_internal.h -- layout of a potential and of the scratch buffers on the
// device, shared by the host code (nnp_host.cpp) and the kernels (nnp_*.cu).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#define NNP_MAX_TYPES 8
#define NNP_MAX_TT (NNP_MAX_TYPES * (NNP_MAX_TYPES + 1) / 2)
#define NNP_MAX_LAYERS 8
#define NNP_MAX_RFUNC 32      // radial functions in one (centre, neighbour) block
#define NNP_MAX_AFUNC 32      // angular functions in one (centre, pair) block
#define NNP_MAX_DAMP 8        // distinct GAUSS damping factors per centre type
#define NNP_MAX_CUT 4         // distinct (cutoff form, rc) pairs in a potential
#define NNP_MAX_NODES 128     // widest network layer handled on the device
#define NNP_MAX_NBR 256       // neighbours per atom staged in shared memory

#ifdef __CUDACC__
#define NNP_HD __host__ __device__
#else
#define NNP_HD
#endif

namespace nnp {

// Row stride of a transposed weight matrix W^T (ni x no) in shared memory:
// odd, so lanes reading a column (fixed n, consecutive m) hit distinct banks.
NNP_HD inline int wt_stride(int no) { return (no % 2 == 0) ? no + 1 : no + 2; }

// Cutoff::Name, BasisR::Name, BasisA::Name, NN::Neuron numbering of the reference
enum CutName { CUT_NONE = 0, CUT_STEP, CUT_COS, CUT_TANH, CUT_POLY3 };
enum RadName { RAD_NONE = 0, RAD_GAUSSIAN, RAD_SECH, RAD_LOGISTIC, RAD_TANH, RAD_LOGCOSH, RAD_LOGCOSH2 };
enum AngName { ANG_NONE = 0, ANG_GAUSS, ANG_GAUSS2, ANG_SECH, ANG_STUDENT3, ANG_STUDENT4, ANG_STUDENT5 };
enum Neuron {
    NEU_NONE = 0, NEU_LINEAR, NEU_SIGMOID, NEU_TANH, NEU_ISRU, NEU_ARCTAN, NEU_RELU, NEU_ELU, NEU_TANHRE,
    NEU_SQRE, NEU_SWISH, NEU_GELU, NEU_MISH, NEU_PFLU, NEU_LOGISH, NEU_SOFTPLUS, NEU_SQPLUS, NEU_ATISH,
    NEU_IERF, NEU_TEST
};

// ---------------------------------------------------------------- host model
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

// ---------------------------------------------------------------- device model
struct DevCut { int name; float rc, rci, pirci; };

struct DevBlockR {
    int n;        // functions
    int off_g;    // offset of the block inside G
    int form;     // RadName
    int cut;      // index into DevPot::cut
    int par;      // first function in rpar (float2: rs, eta)
};

struct DevBlockA {
    int n;
    int off_g;    // absolute offset in G (nInputR + offsetA)
    int form;     // AngName
    int cut;
    int par;      // first function in apar (float4: lambdaf, zeta, ieta2, damp-id|izeta<<8)
    int int_zeta; // all zeta are small non-negative integers -> exact repeated products
};

struct DevType {
    int n_input, n_input_r;
    DevBlockR br[NNP_MAX_TYPES];
    DevBlockA ba[NNP_MAX_TT];
    int ndamp;                      // distinct (cutoff, 1/eta^2) GAUSS damping factors
    float damp_a[NNP_MAX_DAMP];     // 1/eta^2 of the damping factor
    int damp_cut[NNP_MAX_DAMP];     // its cutoff index
    // network
    int nlayer;
    int nodes[NNP_MAX_LAYERS + 1];
    int neuron;
    float c;
    int64_t woff;                   // first float of this network in wpar
};

struct DevPot {
    int ntypes;
    int ncut;
    float rc;
    double rc_d;
    DevCut cut[NNP_MAX_CUT];
    DevType t[NNP_MAX_TYPES];
};

// A network's floats in wpar, starting at DevType::woff:
//   inpw[nin], inpb[nin], outw[nout], outb[nout],
//   then for each layer l: bias[no] and the weights transposed with a padded
//   row, W^T[m * wt_stride(no) + n] = W[n][m]  (m < ni, n < no).
int64_t net_floats(const HostNet &net);

}  // namespace nnp
