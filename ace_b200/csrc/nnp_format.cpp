// nnp_format.cpp -- the reference's potential, basis and network text formats.
//
// read_potential follows NNP::read (src/nnp/nnp.cpp:243-307) line by line:
// "ann", "ntypes N", N type lines (NNH::Type::read, nnh.cpp:65-93), "rc x",
// then per centre type a "basis X" block holding one "basis_radial Y" +
// BasisR block per neighbour type (basis_radial.cpp:123-143) and one
// "basis_angular Y Z" + BasisA block per pair Y<=Z (basis_angular.cpp:116-138),
// then per type "nn X" followed by an ANN block (ml/nn.cpp:1536-1613).
// write_potential reproduces NNP::write (nnp.cpp:197-236) byte for byte.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

#include "nnp_internal.h"

namespace nnp {

int tt_index(int i, int j) { return (i > j) ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

int HostNet::nparams() const
{
    int s = 0;
    for (size_t l = 0; l + 1 < nodes.size(); ++l) s += nodes[l + 1] * (nodes[l] + 1);
    return s;
}

int HostPot::n_input_r(int II) const
{
    int s = 0;
    for (const auto &b : br[II]) s += (int)b.rs.size();
    return s;
}

int HostPot::n_input(int II) const
{
    int s = n_input_r(II);
    for (const auto &b : ba[II]) s += (int)b.eta.size();
    return s;
}

int64_t net_floats(const HostNet &net)
{
    int64_t s = 2 * net.nodes.front() + 2 * net.nodes.back();
    for (size_t l = 0; l + 1 < net.nodes.size(); ++l) s += net.nodes[l + 1] + (int64_t)net.nodes[l] * wt_stride(net.nodes[l + 1]);
    return s;
}

namespace {

const char *kCut[] = {"NONE", "STEP", "COS", "TANH", "POLY3"};
const char *kRad[] = {"NONE", "GAUSSIAN", "SECH", "LOGISTIC", "TANH", "LOGCOSH", "LOGCOSH2"};
const char *kAng[] = {"NONE", "GAUSS", "GAUSS2", "SECH", "STUDENT3", "STUDENT4", "STUDENT5"};
const char *kNeu[] = {"NONE", "LINEAR", "SIGMOID", "TANH", "ISRU", "ARCTAN", "RELU", "ELU", "TANHRE", "SQRE",
                      "SWISH", "GELU", "MISH", "PFLU", "LOGISH", "SOFTPLUS", "SQPLUS", "ATISH", "IERF", "TEST"};

template <size_t N>
int lookup(const char *(&tab)[N], const std::string &s)
{
    for (size_t i = 1; i < N; ++i)
        if (s == tab[i]) return (int)i;
    return 0;
}

struct Lines {
    std::vector<std::string> lines;
    size_t k = 0;
    explicit Lines(const std::string &text)
    {
        std::istringstream is(text);
        std::string ln;
        while (std::getline(is, ln)) lines.push_back(ln);
    }
    bool next(std::vector<std::string> &tok)
    {
        tok.clear();
        if (k >= lines.size()) return false;
        std::istringstream is(lines[k++]);
        std::string t;
        while (is >> t) tok.push_back(t);
        return true;
    }
};

std::string upper(std::string s)
{
    for (auto &c : s) c = (char)toupper((unsigned char)c);
    return s;
}

int name_index(const HostPot &pot, const std::string &n)
{
    for (int i = 0; i < pot.ntypes(); ++i)
        if (pot.types[i].name == n) return i;
    return -1;
}

std::string read_basis_r(Lines &L, HostBasisR &b)
{
    std::vector<std::string> t;
    if (!L.next(t) || t.size() < 5) return "BasisR::read: missing header";
    b.cut = lookup(kCut, t[1]);
    b.rc = std::atof(t[2].c_str());
    b.form = lookup(kRad, t[3]);
    const int n = std::atoi(t[4].c_str());
    if (b.cut == 0) return "Cutoff::Cutoff(Cutoff::Name&,double): Invalid Cutoff name.";
    if (b.rc < 0) return "Cutoff::Cutoff(Cutoff::Name&,double): Invalid Cutoff distance.";
    if (b.form == 0) return "BasisR(rc,Cutoff::Name,int,BasisR::Name): invalid radial function type";
    if (n < 0) return "Basis::resize(int): invalid number of functions.";
    b.rs.resize(n);
    b.eta.resize(n);
    for (int i = 0; i < n; ++i) {
        if (!L.next(t) || t.size() < 2) return "BasisR::read: missing parameter line";
        b.rs[i] = std::atof(t[0].c_str());
        b.eta[i] = std::atof(t[1].c_str());
    }
    return "";
}

std::string read_basis_a(Lines &L, HostBasisA &b)
{
    std::vector<std::string> t;
    if (!L.next(t) || t.size() < 5) return "BasisA::read: missing header";
    b.cut = lookup(kCut, t[1]);
    b.rc = std::atof(t[2].c_str());
    b.form = lookup(kAng, t[3]);
    const int n = std::atoi(t[4].c_str());
    if (b.cut == 0) return "Cutoff::Cutoff(Cutoff::Name&,double): Invalid Cutoff name.";
    if (b.rc < 0) return "Cutoff::Cutoff(Cutoff::Name&,double): Invalid Cutoff distance.";
    if (b.form == 0) return "BasisA(rc,Cutoff::Name,int,BasisA::Name): invalid angular function type";
    if (n < 0) return "Basis::resize(int): invalid number of functions.";
    b.eta.resize(n);
    b.zeta.resize(n);
    b.lambda.resize(n);
    for (int i = 0; i < n; ++i) {
        if (!L.next(t) || t.size() < 3) return "BasisA::read: missing parameter line";
        b.eta[i] = std::atof(t[0].c_str());
        b.zeta[i] = std::atof(t[1].c_str());
        b.lambda[i] = std::atoi(t[2].c_str());
    }
    return "";
}

std::string read_net_lines(Lines &L, HostNet &net)
{
    std::vector<std::string> t;
    if (!L.next(t) || t.size() < 3) return "ANN::read: missing configuration line";
    net.nodes.clear();
    for (size_t i = 1; i < t.size(); ++i) net.nodes.push_back(std::atoi(t[i].c_str()));
    if (net.nodes.size() < 2) return "ANN::resize(const ANNP&,int,const std::vector<int>&): Invalid number of layers.";
    for (int n : net.nodes)
        if (n <= 0) return "ANN::resize(const ANNP&,int,const std::vector<int>&): Invalid layer size.";
    if (net.nodes.back() != 1) return "ANN: the device path supports one network output";
    if (!L.next(t) || t.size() < 3) return "ANN::read: missing neuron line";
    net.neuron = lookup(kNeu, t[1]);
    net.c = std::atof(t[2].c_str());
    if (net.neuron == 0) return "ANN::read(FILE*,ANN&): Invalid neuron.";
    const int nin = net.nodes.front(), nout = net.nodes.back(), nl = (int)net.nodes.size() - 1;
    auto vec = [&](std::vector<double> &v, int n, const char *what) -> std::string {
        if (!L.next(t) || (int)t.size() < n + 1) return std::string("ANN::read: short line ") + what;
        v.resize(n);
        for (int i = 0; i < n; ++i) v[i] = std::atof(t[i + 1].c_str());
        return "";
    };
    std::string e;
    if (!(e = vec(net.inpw, nin, "inpw")).empty()) return e;
    if (!(e = vec(net.outw, nout, "outw")).empty()) return e;
    if (!(e = vec(net.inpb, nin, "inpb")).empty()) return e;
    if (!(e = vec(net.outb, nout, "outb")).empty()) return e;
    net.b.assign(nl, {});
    net.w.assign(nl, {});
    for (int l = 0; l < nl; ++l)
        if (!(e = vec(net.b[l], net.nodes[l + 1], "bias")).empty()) return e;
    for (int l = 0; l < nl; ++l)
        if (!(e = vec(net.w[l], net.nodes[l + 1] * net.nodes[l], "weight")).empty()) return e;
    return "";
}

void appendf(std::string &s, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
void appendf(std::string &s, const char *fmt, ...)
{
    char buf[256];
    va_list ap;
    va_start(ap, fmt);
    int n = vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (n >= (int)sizeof buf) {
        std::vector<char> big(n + 1);
        va_start(ap, fmt);
        vsnprintf(big.data(), big.size(), fmt, ap);
        va_end(ap);
        s += big.data();
    } else {
        s += buf;
    }
}

// BasisA::init rflag grouping (basis_angular.cpp:184-197), for writing
std::vector<int> rflag_of(const HostBasisA &b)
{
    std::vector<int> r(b.eta.size(), 0);
    int flag = 0;
    for (size_t n = 1; n < b.eta.size(); ++n) {
        if (std::fabs(b.eta[n] - b.eta[n - 1]) >= 1.0e-6) ++flag;
        r[n] = flag;
    }
    return r;
}

}  // namespace

std::string read_network(const std::string &text, HostNet &net)
{
    Lines L(text);
    return read_net_lines(L, net);
}

std::string read_potential(const std::string &text, HostPot &pot)
{
    Lines L(text);
    std::vector<std::string> t;
    pot = HostPot();
    if (!L.next(t)) return "NNP::read: empty file";                       // header
    if (!L.next(t) || t.size() < 2) return "NNP::read: missing ntypes";
    const int T = std::atoi(t[1].c_str());
    if (T <= 0) return "NNP::read(FILE*,NNP&): invalid number of types.";
    if (T > NNP_MAX_TYPES) return "NNP::read: more element types than the device path supports";
    pot.types.resize(T);
    for (int n = 0; n < T; ++n) {
        if (!L.next(t)) return "NNP::read: missing type line";
        HostType &ty = pot.types[n];
        ty.name = "NONE";
        for (size_t k = 0; k < t.size();) {
            const std::string tag = upper(t[k++]);
            if (k >= t.size()) break;
            const std::string &v = t[k];
            double *f = nullptr;
            if (tag == "NAME") { ty.name = v; ++k; continue; }
            if (tag == "ENERGY") f = &ty.energy;
            else if (tag == "MASS") f = &ty.mass;
            else if (tag == "CHARGE") f = &ty.charge;
            else if (tag == "RADIUS") f = &ty.radius;
            else if (tag == "Z") f = &ty.z;
            else if (tag == "ALPHA") f = &ty.alpha;
            else if (tag == "IE") f = &ty.ie;
            else if (tag == "RCOV") f = &ty.rcov;
            else if (tag == "RVDW") f = &ty.rvdw;
            else if (tag == "AMP") f = &ty.amp;
            if (f) { *f = std::atof(v.c_str()); ++k; }
        }
    }
    if (!L.next(t) || t.size() < 2) return "NNP::read: missing rc";
    pot.rc = std::atof(t[1].c_str());
    if (pot.rc <= 0) return "NNP::read(FILE*,NNP&): invalid cutoff.";
    const int TT = T * (T + 1) / 2;
    pot.br.assign(T, std::vector<HostBasisR>(T));
    pot.ba.assign(T, std::vector<HostBasisA>(TT));
    for (int i = 0; i < T; ++i) {
        if (!L.next(t) || t.size() < 2) return "NNP::read: missing basis line";
        const int II = name_index(pot, t[1]);
        if (II < 0) return "NNP::read: unknown type " + t[1];
        for (int j = 0; j < T; ++j) {
            if (!L.next(t) || t.size() < 2) return "NNP::read: missing basis_radial line";
            const int JJ = name_index(pot, t[1]);
            if (JJ < 0) return "NNP::read: unknown type " + t[1];
            std::string e = read_basis_r(L, pot.br[II][JJ]);
            if (!e.empty()) return e;
        }
        for (int j = 0; j < TT; ++j) {
            if (!L.next(t) || t.size() < 3) return "NNP::read: missing basis_angular line";
            const int JJ = name_index(pot, t[1]), KK = name_index(pot, t[2]);
            if (JJ < 0 || KK < 0) return "NNP::read: unknown type in basis_angular";
            std::string e = read_basis_a(L, pot.ba[II][tt_index(JJ, KK)]);
            if (!e.empty()) return e;
        }
    }
    pot.nets.assign(T, HostNet());
    for (int n = 0; n < T; ++n) {
        if (!L.next(t) || t.size() < 2) return "NNP::read: missing nn line";
        const int II = name_index(pot, t[1]);
        if (II < 0) return "NNP::read: unknown type " + t[1];
        std::string e = read_net_lines(L, pot.nets[II]);
        if (!e.empty()) return e;
    }
    for (int II = 0; II < T; ++II)
        if (pot.nets[II].nodes.front() != pot.n_input(II))
            return "NNP::read: network input size differs from the basis size of " + pot.types[II].name;
    return "";
}

// NNP::read_basis (nnp.cpp:113-156): "<tag> rc", "<tag> ntypes", "<tag> centre",
// then radial and angular blocks for the centre type II.
std::string read_basis_file(const std::string &text, HostPot &pot, int II)
{
    Lines L(text);
    std::vector<std::string> t;
    if (!L.next(t) || t.size() < 2) return "NNP::read_basis: missing cutoff";
    if (std::atof(t[1].c_str()) != pot.rc) return "NNP::read_basis(FILE*,NNP&,const char*): invalid cutoff.";
    if (!L.next(t) || t.size() < 2) return "NNP::read_basis: missing ntypes";
    const int T = std::atoi(t[1].c_str());
    if (T != pot.ntypes()) return "NNP::read_basis(FILE*,NNP&,const char*): invalid number of types.";
    if (!L.next(t) || t.size() < 2) return "NNP::read_basis: missing central type";
    if (name_index(pot, t[1]) != II) return "NNP::read_basis(FILE*,NNP&,const char*): invalid central types.";
    for (int j = 0; j < T; ++j) {
        if (!L.next(t) || t.size() < 2) return "NNP::read_basis: missing radial type line";
        const int JJ = name_index(pot, t[1]);
        if (JJ < 0) return "NNP::read_basis: unknown type " + t[1];
        std::string e = read_basis_r(L, pot.br[II][JJ]);
        if (!e.empty()) return e;
    }
    for (int j = 0; j < T; ++j)
        for (int k = j; k < T; ++k) {
            if (!L.next(t) || t.size() < 3) return "NNP::read_basis: missing angular type line";
            const int JJ = name_index(pot, t[1]), KK = name_index(pot, t[2]);
            if (JJ < 0 || KK < 0) return "NNP::read_basis: unknown type in angular line";
            std::string e = read_basis_a(L, pot.ba[II][tt_index(JJ, KK)]);
            if (!e.empty()) return e;
        }
    return "";
}

std::string write_potential(const HostPot &pot)
{
    std::string s;
    const int T = pot.ntypes();
    s += "ann\n";
    appendf(s, "ntypes %i\n", T);
    for (const auto &ty : pot.types) {       // NNH::Type::write (nnh.cpp:95-108)
        appendf(s, "name %s ", ty.name.c_str());
        appendf(s, "energy %f ", ty.energy);
        appendf(s, "mass %f ", ty.mass);
        appendf(s, "charge %f ", ty.charge);
        appendf(s, "radius %f ", ty.radius);
        appendf(s, "z %f ", ty.z);
        appendf(s, "alpha %f ", ty.alpha);
        appendf(s, "ie %f ", ty.ie);
        appendf(s, "rcov %f ", ty.rcov);
        appendf(s, "rvdw %f ", ty.rvdw);
        appendf(s, "amp %f ", ty.amp);
        s += "\n";
    }
    appendf(s, "rc %f\n", pot.rc);
    for (int i = 0; i < T; ++i) {
        appendf(s, "basis %s\n", pot.types[i].name.c_str());
        for (int j = 0; j < T; ++j) {
            appendf(s, "basis_radial %s\n", pot.types[j].name.c_str());
            const HostBasisR &b = pot.br[i][j];
            appendf(s, "BasisR %s %f %s %i\n", kCut[b.cut], b.rc, kRad[b.form], (int)b.rs.size());
            for (size_t n = 0; n < b.rs.size(); ++n) appendf(s, "\t%f %f\n", b.rs[n], b.eta[n]);
        }
        for (int j = 0; j < T; ++j)
            for (int k = j; k < T; ++k) {
                appendf(s, "basis_angular %s %s\n", pot.types[j].name.c_str(), pot.types[k].name.c_str());
                const HostBasisA &b = pot.ba[i][tt_index(j, k)];
                appendf(s, "BasisA %s %f %s %i\n", kCut[b.cut], b.rc, kAng[b.form], (int)b.eta.size());
                const std::vector<int> rf = rflag_of(b);
                for (size_t n = 0; n < b.eta.size(); ++n)
                    appendf(s, "\t%f %f %i %i\n", b.eta[n], b.zeta[n], b.lambda[n], rf[n]);
            }
    }
    for (int n = 0; n < T; ++n) {            // ANN::write (ml/nn.cpp:1471-1511)
        appendf(s, "nn %s\n", pot.types[n].name.c_str());
        const HostNet &net = pot.nets[n];
        appendf(s, "nn %i ", net.nodes.front());
        for (size_t l = 1; l < net.nodes.size(); ++l) appendf(s, "%i ", net.nodes[l]);
        s += "\n";
        appendf(s, "neuron %s %f\n", kNeu[net.neuron], net.c);
        s += "inpw ";
        for (double v : net.inpw) appendf(s, "%.15f ", v);
        s += "\noutw ";
        for (double v : net.outw) appendf(s, "%.15f ", v);
        s += "\ninpb ";
        for (double v : net.inpb) appendf(s, "%.15f ", v);
        s += "\noutb ";
        for (double v : net.outb) appendf(s, "%.15f ", v);
        s += "\n";
        for (size_t l = 0; l < net.b.size(); ++l) {
            appendf(s, "bias[%i] ", (int)l + 1);
            for (double v : net.b[l]) appendf(s, "%.15f ", v);
            s += "\n";
        }
        for (size_t l = 0; l < net.w.size(); ++l) {
            appendf(s, "weight[%i,%i] ", (int)l, (int)l + 1);
            for (double v : net.w[l]) appendf(s, "%.15f ", v);
            s += "\n";
        }
    }
    return s;
}

}  // namespace nnp
