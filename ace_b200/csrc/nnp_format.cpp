// nnp_format.cpp -- the reference's potential, basis and network text formats.
//
// read_potential follows NNP::read (src/nnp/nnp.cpp:243-307) line by line:
// "ann", "ntypes N", N type lines (NNH::Type::read, nnh.cpp:65-93), "rc x",
// then per centre type a "basis X" block holding one "basis_radial Y" +
// BasisR block per neighbour type (basis_radial.cpp:123-143) and one
// "basis_angular Y Z" + BasisA block per pair Y<=Z (basis_angular.cpp:116-138),
// then per type "nn X" followed by an ANN block (ml/nn.cpp:1536-1613).
// write_potential reproduces NNP::write (nnp.cpp:197-236) byte for byte.
#include <algorithm>
#include <cctype>
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

// ------------------------------------------------------------------ structure files
//
// Readers of the structure formats the reference's training and test
// programs take (format/xyz_struc.cpp, format/vasp_struc.cpp), into the CSR
// batch of the C ABI, in the reference's METAL units (A, eV).

namespace nnp {

namespace {

std::vector<std::string> split_ws(const std::string &s)
{
    std::vector<std::string> out;
    std::istringstream is(s);
    std::string t;
    while (is >> t) out.push_back(t);
    return out;
}

// value text after "KEY=" in an extended-XYZ comment line (quotes removed)
bool xyz_field(const std::string &line, const std::string &key, std::string &val)
{
    const std::string up = upper(line);
    const size_t k = up.find(key);
    if (k == std::string::npos) return false;
    size_t p = k + key.size();
    while (p < line.size() && (line[p] == ' ' || line[p] == '=' || line[p] == '\t')) ++p;
    if (p < line.size() && line[p] == '"') {
        const size_t e = line.find('"', p + 1);
        val = line.substr(p + 1, e == std::string::npos ? std::string::npos : e - p - 1);
    } else {
        size_t e = p;
        while (e < line.size() && !std::isspace((unsigned char)line[e])) ++e;
        val = line.substr(p, e - p);
    }
    return true;
}

// positions back into the cell, Cell::returnToCell (struc/cell.cpp): fractional
// coordinates reduced to [0, 1)
void wrap_into_cell(const double R[9], double *x)
{
    // R[3n + d] = component d of lattice vector n; solve R q = x
    const double *a = R, *b = R + 3, *c = R + 6;
    const double bc[3] = {b[1] * c[2] - b[2] * c[1], b[2] * c[0] - b[0] * c[2], b[0] * c[1] - b[1] * c[0]};
    const double ca[3] = {c[1] * a[2] - c[2] * a[1], c[2] * a[0] - c[0] * a[2], c[0] * a[1] - c[1] * a[0]};
    const double ab[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    const double V = a[0] * bc[0] + a[1] * bc[1] + a[2] * bc[2];
    if (!(std::fabs(V) > 0)) return;
    double q[3] = {(bc[0] * x[0] + bc[1] * x[1] + bc[2] * x[2]) / V, (ca[0] * x[0] + ca[1] * x[1] + ca[2] * x[2]) / V,
                   (ab[0] * x[0] + ab[1] * x[1] + ab[2] * x[2]) / V};
    for (double &v : q) v -= std::floor(v);
    for (int d = 0; d < 3; ++d) x[d] = R[d] * q[0] + R[3 + d] * q[1] + R[6 + d] * q[2];
}

}  // namespace

// Extended XYZ (every frame of the file): line 1 the atom count, line 2
// Properties=species:S:1:pos:R:3[:forces:R:3...], potential_energy=E and
// Lattice="a1 a2 a3" (vectors in turn), then one line per atom
// (XYZ::read, format/xyz_struc.cpp:26-180).  Without a Properties field the
// atom lines are "name x y z".  A frame with a lattice is periodic and its
// positions are wrapped into the cell, as the reference does.
std::string read_xyz_frames(const std::string &text, std::vector<ReadStruct> &out)
{
    std::istringstream in(text);
    std::string line;
    while (std::getline(in, line)) {
        const std::vector<std::string> t0 = split_ws(line);
        if (t0.empty()) continue;
        char *end = nullptr;
        const long n = std::strtol(t0[0].c_str(), &end, 10);
        if (!end || *end || n <= 0) return "XYZ: expected an atom count, found \"" + line + "\"";
        std::string head;
        if (!std::getline(in, head)) return "XYZ: missing comment line";
        ReadStruct rs;
        rs.pbc = false;
        rs.energy = 0.0;
        std::fill(rs.cell, rs.cell + 9, 0.0);
        // columns of the atom lines
        int ndata = 0, ni = 0, ri = 1, fi = -1;
        std::string props;
        if (xyz_field(head, "PROPERTIES", props)) {
            ni = ri = -1;
            std::vector<std::string> f;
            std::string cur;
            for (char c : props) {
                if (c == ':') { f.push_back(cur); cur.clear(); }
                else cur += c;
            }
            f.push_back(cur);
            for (size_t k = 0; k + 2 < f.size(); k += 3) {
                const std::string tag = upper(f[k]);
                const int len = std::atoi(f[k + 2].c_str());
                if (tag == "SPECIES") ni = ndata;
                else if (tag == "POS" || tag == "POSN" || tag == "POSITION") ri = ndata;
                else if (tag == "FORCES" || tag == "FORCE") fi = ndata;
                ndata += len;
            }
            if (ni < 0 || ri < 0) return "XYZ: Properties without species and positions";
        }
        std::string v;
        if (xyz_field(head, "POTENTIAL_ENERGY", v)) rs.energy = std::atof(v.c_str());
        if (xyz_field(head, "LATTICE", v)) {
            const std::vector<std::string> L = split_ws(v);
            if (L.size() != 9) return "XYZ: Lattice needs 9 numbers";
            double nrm = 0;
            for (int k = 0; k < 9; ++k) {
                rs.cell[k] = std::atof(L[k].c_str());
                nrm += rs.cell[k] * rs.cell[k];
            }
            rs.pbc = nrm > 0;
        }
        rs.has_forces = fi >= 0;
        for (long i = 0; i < n; ++i) {
            if (!std::getline(in, line)) return "XYZ: fewer atom lines than the atom count";
            const std::vector<std::string> a = split_ws(line);
            const int need = std::max({ni + 1, ri + 3, fi >= 0 ? fi + 3 : 0});
            if ((int)a.size() < need) return "XYZ: short atom line \"" + line + "\"";
            rs.names.push_back(a[ni]);
            double x[3] = {std::atof(a[ri].c_str()), std::atof(a[ri + 1].c_str()), std::atof(a[ri + 2].c_str())};
            if (rs.pbc) wrap_into_cell(rs.cell, x);
            rs.pos.insert(rs.pos.end(), x, x + 3);
            for (int d = 0; d < 3; ++d) rs.forces.push_back(fi >= 0 ? std::atof(a[fi + d].c_str()) : 0.0);
        }
        out.push_back(std::move(rs));
    }
    return "";
}

// VASP POSCAR / CONTCAR (VASP::POSCAR::read, format/vasp_struc.cpp:41-190): comment,
// scale, three lattice vectors (times the scale), species names, counts,
// "Direct" or Cartesian, positions.  As in the reference, Cartesian positions
// are taken as they stand (the scale multiplies the lattice only).
std::string read_vasp(const std::string &text, std::vector<ReadStruct> &out)
{
    std::istringstream in(text);
    std::string line;
    auto next = [&](std::string &l) { return (bool)std::getline(in, l); };
    ReadStruct rs;
    if (!next(line)) return "VASP: empty file";
    if (!next(line)) return "VASP: missing scale";
    const double scale = std::atof(line.c_str());
    for (int n = 0; n < 3; ++n) {
        if (!next(line)) return "VASP: missing lattice vector";
        const std::vector<std::string> v = split_ws(line);
        if (v.size() < 3) return "VASP: short lattice vector";
        for (int d = 0; d < 3; ++d) rs.cell[3 * n + d] = std::atof(v[d].c_str()) * scale;
    }
    std::string sn, sc;
    if (!next(sn) || !next(sc)) return "VASP: missing species";
    const std::vector<std::string> names = split_ws(sn), counts = split_ws(sc);
    if (names.empty() || names.size() != counts.size()) return "Invalid number of species";
    if (!next(line)) return "VASP: missing coordinate mode";
    const bool direct = !line.empty() && line[0] == 'D';
    for (size_t s = 0; s < names.size(); ++s) {
        const int c = std::atoi(counts[s].c_str());
        for (int m = 0; m < c; ++m) {
            if (!next(line)) return "VASP: fewer positions than atoms";
            const std::vector<std::string> v = split_ws(line);
            if (v.size() < 3) return "VASP: short position line";
            double x[3] = {std::atof(v[0].c_str()), std::atof(v[1].c_str()), std::atof(v[2].c_str())};
            if (direct) {
                const double q[3] = {x[0], x[1], x[2]};
                for (int d = 0; d < 3; ++d) x[d] = rs.cell[d] * q[0] + rs.cell[3 + d] * q[1] + rs.cell[6 + d] * q[2];
            }
            rs.pos.insert(rs.pos.end(), x, x + 3);
            rs.names.push_back(names[s]);
            for (int d = 0; d < 3; ++d) rs.forces.push_back(0.0);
        }
    }
    rs.pbc = true;
    rs.energy = 0.0;
    rs.has_forces = false;
    out.push_back(std::move(rs));
    return "";
}

}  // namespace nnp
