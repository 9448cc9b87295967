// emu_host.cpp -- host-side parts of the C ABI: the inputs-file reader
// (TestParams::Initialize, Source/Parameters.H:52-131), initial conditions
// (FlavoredNeutrinoContainer::InitParticles,
// Source/FlavoredNeutrinoContainerInit.cpp:9-661), the vacuum mass matrix,
// and the AMReX plotfile / particle-checkpoint writer and reader
// (Source/IO.cpp:11-63; layout read by Scripts/tests/EmuReader.py:19-113).
#include "emu_host.h"

#include <sys/stat.h>
#include <sys/types.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

const double kEV = 1.60218e-12;
const double kC = 2.99792458e10;
const double kHbar = 1.05457266e-27;

int herm_re(int nf, int i, int j)
{
    int base = 0;
    for (int r = 0; r < i; r++) base += 1 + 2 * (nf - 1 - r);
    return base + (j == i ? 0 : 1 + 2 * (j - i - 1));
}

double su_length(int nf, const double* f)
{
    double s = 0.0;
    for (int i = 0; i < nf; i++)
        for (int j = i + 1; j < nf; j++) {
            double a = f[herm_re(nf, i, j) + 1], b = f[herm_re(nf, i, j)];
            s = s + a * a;
            s = s + b * b;
        }
    for (int l = 1; l < nf; l++) {
        double cl = std::sqrt(2.0 / (l * (l + 1.0))) / 2.0;
        double t = 0.0;
        for (int i = 0; i < l; i++) t = t + cl * f[herm_re(nf, i, i)];
        t = t - (cl * l) * f[herm_re(nf, l, l)];
        s = s + t * t;
    }
    return std::sqrt(s);
}

}  // namespace

namespace emu_host {

double c2() { return kC * kC; }
double c4() { return c2() * c2(); }
double hbarc() { return kHbar * kC; }
double gf()
{
    const double hc = hbarc();
    return 1.1663787e-5 / (1e9 * 1e9 * kEV * kEV) * hc * hc * hc;
}

bool validate(const emu_params& p, std::string& why)
{
    if (p.nflavors != 2 && p.nflavors != 3) { why = "nflavors must be 2 or 3"; return false; }
    if (p.shape_order < 0 || p.shape_order > 2) { why = "shape_order must be 0, 1 or 2"; return false; }
    if (p.precision != EMU_PREC_FP64 && p.precision != EMU_PREC_MIXED) { why = "precision must be 0 or 1"; return false; }
    for (int d = 0; d < 3; d++) {
        if (p.ncell[d] < 1) { why = "ncell must be >= 1"; return false; }
        const int ord = p.ncell[d] > 1 ? p.shape_order : 0;
        const int ngrow = 1 + (1 + ord) / 2;            // main.cpp:68-72
        if (p.ncell[d] < ngrow) { why = "ncell smaller than the ghost width (main.cpp:72)"; return false; }
    }
    const long long nc = (long long)p.ncell[0] * p.ncell[1] * p.ncell[2];
    if (nc >= (1ll << 31)) { why = "more than 2^31 cells"; return false; }
    if (!(p.Lx > 0 && p.Ly > 0 && p.Lz > 0)) { why = "domain lengths must be positive"; return false; }
    if (p.precision == EMU_PREC_MIXED && !(p.integration_type == 1 && p.rk_type == 4)) {
        why = "the mixed-precision path integrates with RK4 (integration.type=1, integration.rk.type=4)";
        return false;
    }
    if (p.integration_type != 0 && p.integration_type != 1) { why = "integration.type must be 0 or 1"; return false; }
    if (p.integration_type == 1 && (p.rk_type < 2 || p.rk_type > 4)) {
        why = "integration.rk.type must be 2, 3 or 4";
        return false;
    }
    return true;
}

void vacuum_m2(const emu_params& p, double m2[2][9])
{
    using cd = std::complex<double>;
    const int nf = p.nflavors;
    cd U[3][3] = {}, R12[3][3] = {}, R13[3][3] = {}, R23[3][3] = {}, A[3][3] = {};
    for (int i = 0; i < nf; i++) R12[i][i] = R13[i][i] = R23[i][i] = 1.0;
    R12[0][0] = std::cos(p.theta12);
    R12[0][1] = std::sin(p.theta12);
    R12[1][0] = -std::sin(p.theta12);
    R12[1][1] = std::cos(p.theta12);
    if (nf == 2) {
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++) U[i][j] = R12[i][j];
    } else {
        // U23 built from theta13, as generate_code.py:202-209 does
        const double s13 = std::sin(p.theta13), c13 = std::cos(p.theta13);
        R13[0][0] = c13;
        R13[0][2] = s13 * cd(std::cos(-p.deltaCP), std::sin(-p.deltaCP));
        R13[2][0] = -s13 * cd(std::cos(p.deltaCP), std::sin(p.deltaCP));
        R13[2][2] = c13;
        R23[0][0] = c13;
        R23[0][2] = s13;
        R23[2][0] = -s13;
        R23[2][2] = c13;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                cd s = 0;
                for (int k = 0; k < 3; k++) s += R23[i][k] * R13[k][j];
                A[i][j] = s;
            }
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                cd s = 0;
                for (int k = 0; k < 3; k++) s += A[i][k] * R12[k][j];
                U[i][j] = s;
            }
    }
    // the Majorana phase matrix commutes with diag(m^2) and cancels
    const double m[3] = {p.mass1 * p.mass1, p.mass2 * p.mass2, p.mass3 * p.mass3};
    for (int s = 0; s < 2; s++)
        for (int e = 0; e < 9; e++) m2[s][e] = 0.0;
    for (int i = 0; i < nf; i++)
        for (int j = i; j < nf; j++) {
            cd v = 0;
            for (int k = 0; k < nf; k++) v += U[i][k] * m[k] * std::conj(U[j][k]);
            const int e = herm_re(nf, i, j);
            m2[0][e] = v.real();
            m2[1][e] = v.real();
            if (j > i) {
                m2[0][e + 1] = v.imag();
                m2[1][e + 1] = -v.imag();
            }
        }
}

void weight_totals(const emu_params& p, const double* records, long long n, double total[2], double mx[2])
{
    const int nf = p.nflavors, nh = nf * nf, nr = 3 + 8 + 2 * (2 + nh);
    for (int s = 0; s < 2; s++) {
        total[s] = mx[s] = 0.0;
        const int off = 3 + 8 + s * (2 + nh);
        for (long long i = 0; i < n; i++) {
            const double v = std::fabs(records[i * nr + off]);
            total[s] += v;
            if (v > mx[s]) mx[s] = v;
        }
    }
}

bool fixed_point_scales(const emu_params& p, const double* records, long long n, double scale[2], double unscale[2],
                        std::string& why)
{
    double total[2], mx[2];
    weight_totals(p, records, n, total, mx);
    return fixed_point_scales_from(total, mx, scale, unscale, why);
}

bool fixed_point_scales_from(const double totals[2], const double maxima[2], double scale[2], double unscale[2],
                             std::string& why)
{
    for (int s = 0; s < 2; s++) {
        const double total = totals[s], mx = maxima[s];
        if (mx > 1e37) {
            why = "particle weight N above 1e37 does not fit the FP32 arithmetic of the mixed path";
            return false;
        }
        // a cell sum of |w f N v| is below 2*total (|f_ij| <= 1 with margin, |v| <= 1)
        const double bound = 2.0 * total;
        int k = 0;
        if (bound > 0) k = 61 - (int)std::ceil(std::log2(bound));
        if (k > 120) k = 120;
        if (k < -120) k = -120;
        scale[s] = std::ldexp(1.0, k);
        unscale[s] = std::ldexp(1.0, -k);
    }
    return true;
}

// ---- plotfile writer ---------------------------------------------------------
static bool mkdir_p(const std::string& d)
{
    std::string cur;
    for (size_t i = 0; i <= d.size(); i++) {
        if (i == d.size() || d[i] == '/') {
            if (!cur.empty() && mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST) return false;
        }
        if (i < d.size()) cur += d[i];
    }
    return true;
}

std::vector<std::string> grid_names(int nf)
{
    // GIdx::Initialize (Evolve.cpp:8-20) + generated grid_names fill
    std::vector<std::string> names = {"rho", "T", "Ye"};
    const char* vars[4] = {"N", "Fx", "Fy", "Fz"};
    const char* tails[2] = {"", "bar"};
    for (int v = 0; v < 4; v++)
        for (int t = 0; t < 2; t++)
            for (int i = 0; i < nf; i++)
                for (int j = i; j < nf; j++) {
                    names.push_back(std::string(vars[v]) + std::to_string(i) + std::to_string(j) + "_Re" + tails[t]);
                    if (j > i)
                        names.push_back(std::string(vars[v]) + std::to_string(i) + std::to_string(j) + "_Im" +
                                        tails[t]);
                }
    return names;
}

std::vector<std::string> particle_names(int nf)
{
    // FlavoredNeutrinoContainerInit.H_particle_varnames_fill
    std::vector<std::string> names = {"time", "x", "y", "z", "pupx", "pupy", "pupz", "pupt"};
    const char* tails[2] = {"", "bar"};
    for (int t = 0; t < 2; t++) {
        names.push_back(std::string("N") + tails[t]);
        names.push_back(std::string("L") + tails[t]);
        for (int i = 0; i < nf; i++)
            for (int j = i; j < nf; j++) {
                names.push_back("f" + std::to_string(i) + std::to_string(j) + "_Re" + tails[t]);
                if (j > i) names.push_back("f" + std::to_string(i) + std::to_string(j) + "_Im" + tails[t]);
            }
    }
    return names;
}

static std::string fmt17(double v)
{
    char b[64];
    std::snprintf(b, sizeof b, "%.17g", v);
    return b;
}

bool write_plotfile(const emu_params& p, const char* dir, double time, int step, const double* mesh,
                    const double* records, long long n, std::string& why)
{
    const int nf = p.nflavors;
    const std::string root(dir);
    if (!mkdir_p(root + "/Level_0")) { why = "cannot create " + root; return false; }
    const std::vector<std::string> names = grid_names(nf);
    const int ncomp = (int)names.size();
    const int nx = p.ncell[0], ny = p.ncell[1], nz = p.ncell[2];
    const long long nc = (long long)nx * ny * nz;
    const double L[3] = {p.Lx, p.Ly, p.Lz};
    // single-level plotfile header (WriteSingleLevelPlotfile layout)
    {
        std::ofstream h(root + "/Header");
        if (!h) { why = "cannot write Header"; return false; }
        h << "HyperCLaw-V1.1\n" << ncomp << "\n";
        for (auto& s : names) h << s << "\n";
        h << 3 << "\n" << fmt17(time) << "\n" << 0 << "\n";
        h << "0 0 0\n" << fmt17(L[0]) << " " << fmt17(L[1]) << " " << fmt17(L[2]) << "\n";
        h << "\n";
        h << "((0,0,0) (" << nx - 1 << "," << ny - 1 << "," << nz - 1 << ") (0,0,0))\n";
        h << step << "\n";
        h << fmt17(L[0] / nx) << " " << fmt17(L[1] / ny) << " " << fmt17(L[2] / nz) << "\n";
        h << 0 << "\n" << 0 << "\n";
        h << 0 << " " << 1 << " " << fmt17(time) << "\n" << step << "\n";
        for (int d = 0; d < 3; d++) h << fmt17(0.0) << " " << fmt17(L[d]) << "\n";
        h << "Level_0/Cell\n";
    }
    // one FAB holding every component, FP64 little endian
    std::string fabhdr;
    {
        std::ostringstream f;
        f << "FAB ((8, (64 11 52 0 1 12 0 1023)),(8, (1 2 3 4 5 6 7 8)))";
        f << "((0,0,0) (" << nx - 1 << "," << ny - 1 << "," << nz - 1 << ") (0,0,0)) " << ncomp << "\n";
        fabhdr = f.str();
        std::ofstream d(root + "/Level_0/Cell_D_00000", std::ios::binary);
        if (!d) { why = "cannot write Cell_D_00000"; return false; }
        d << fabhdr;
        d.write(reinterpret_cast<const char*>(mesh), sizeof(double) * nc * ncomp);
    }
    {
        std::ofstream h(root + "/Level_0/Cell_H");
        h << "1\n1\n" << ncomp << "\n0\n";
        h << "(1 0\n((0,0,0) (" << nx - 1 << "," << ny - 1 << "," << nz - 1 << ") (0,0,0))\n)\n";
        h << "1\nFabOnDisk: Cell_D_00000 0\n\n";
        h << "1," << ncomp << "\n";
        for (int c = 0; c < ncomp; c++) {
            double mn = mesh[(long long)c * nc];
            for (long long i = 0; i < nc; i++) mn = std::min(mn, mesh[(long long)c * nc + i]);
            h << fmt17(mn) << ",";
        }
        h << "\n\n1," << ncomp << "\n";
        for (int c = 0; c < ncomp; c++) {
            double mx = mesh[(long long)c * nc];
            for (long long i = 0; i < nc; i++) mx = std::max(mx, mesh[(long long)c * nc + i]);
            h << fmt17(mx) << ",";
        }
        h << "\n";
    }
    if (records) {
        // particle checkpoint pltNNNNN/neutrinos (ParticleContainer::Checkpoint
        // with is_checkpoint = true): ints (id, cpu) then reals (pos + rdata)
        const std::string pdir = root + "/neutrinos";
        if (!mkdir_p(pdir + "/Level_0")) { why = "cannot create " + pdir; return false; }
        const std::vector<std::string> pn = particle_names(nf);
        const int nreal = 3 + (int)pn.size();
        {
            std::ofstream d(pdir + "/Level_0/DATA_00000", std::ios::binary);
            if (!d) { why = "cannot write DATA_00000"; return false; }
            std::vector<int32_t> ints((size_t)n * 2);
            for (long long i = 0; i < n; i++) {
                ints[2 * i] = (int32_t)(i + 1);
                ints[2 * i + 1] = 0;
            }
            d.write(reinterpret_cast<const char*>(ints.data()), sizeof(int32_t) * ints.size());
            d.write(reinterpret_cast<const char*>(records), sizeof(double) * (size_t)n * nreal);
        }
        std::ofstream h(pdir + "/Header");
        h << "Version_Two_Dot_Zero_double\n3\n" << pn.size() << "\n";
        for (auto& s : pn) h << s << "\n";
        h << 0 << "\n" << 1 << "\n" << n << "\n" << n + 1 << "\n" << 0 << "\n" << 1 << "\n";
        h << 0 << " " << n << " " << 0 << "\n";
        std::ofstream ph(pdir + "/Level_0/Particle_H");
        ph << "(1 0\n((0,0,0) (" << nx - 1 << "," << ny - 1 << "," << nz - 1 << ") (0,0,0))\n)\n";
    }
    {
        std::ofstream j(root + "/job_info");
        j << "emu_b200 plotfile\nnflavors: " << nf << "\nstep: " << step << "\ntime: " << fmt17(time) << "\n";
    }
    return true;
}

}  // namespace emu_host

// ===========================================================================
// inputs-file reader
// ===========================================================================
namespace {

struct Inputs {
    std::map<std::string, std::vector<std::string>> kv;
};

std::string trim(const std::string& s)
{
    size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

// ParmParse value list: whitespace separated tokens, "(a, b, c)" tuples are
// one token each, quoted strings keep their spaces
std::vector<std::string> tokens(const std::string& v)
{
    std::vector<std::string> out;
    size_t i = 0;
    while (i < v.size()) {
        while (i < v.size() && std::isspace((unsigned char)v[i])) i++;
        if (i >= v.size()) break;
        if (v[i] == '"') {
            size_t j = v.find('"', i + 1);
            if (j == std::string::npos) j = v.size();
            out.push_back(v.substr(i + 1, j - i - 1));
            i = j + 1;
        } else if (v[i] == '(') {
            size_t j = v.find(')', i);
            if (j == std::string::npos) j = v.size() - 1;
            out.push_back(v.substr(i, j - i + 1));
            i = j + 1;
        } else {
            size_t j = i;
            while (j < v.size() && !std::isspace((unsigned char)v[j])) j++;
            out.push_back(v.substr(i, j - i));
            i = j;
        }
    }
    return out;
}

bool add_line(Inputs& in, const std::string& raw)
{
    std::string line = raw;
    // strip comments outside quotes
    bool q = false;
    for (size_t i = 0; i < line.size(); i++) {
        if (line[i] == '"') q = !q;
        if (line[i] == '#' && !q) { line = line.substr(0, i); break; }
    }
    line = trim(line);
    if (line.empty()) return true;
    size_t eq = line.find('=');
    if (eq == std::string::npos) return false;
    std::string key = trim(line.substr(0, eq));
    std::vector<std::string> val = tokens(line.substr(eq + 1));
    in.kv[key] = val;   // later definitions (and command-line overrides) win
    return true;
}

struct Getter {
    const Inputs& in;
    std::string missing;
    bool has(const char* k) const { return in.kv.count(k) && !in.kv.at(k).empty(); }
    std::string str(const char* k)
    {
        if (!in.kv.count(k)) { if (missing.empty()) missing = k; return std::string(); }
        const auto& v = in.kv.at(k);
        return v.empty() ? std::string() : v[0];
    }
    double d(const char* k)
    {
        std::string s = str(k);
        return s.empty() ? 0.0 : std::strtod(s.c_str(), nullptr);
    }
    int i(const char* k)
    {
        std::string s = str(k);
        if (s == "true") return 1;
        if (s == "false") return 0;
        return s.empty() ? 0 : (int)std::strtol(s.c_str(), nullptr, 10);
    }
    void ivec(const char* k, int out[3])
    {
        std::string s = str(k);
        std::string t;
        for (char ch : s)
            if (ch != '(' && ch != ')') t += (ch == ',' ? ' ' : ch);
        std::istringstream is(t);
        for (int a = 0; a < 3; a++) is >> out[a];
    }
    double d_or(const char* k, double def) { return has(k) ? d(k) : def; }
    int i_or(const char* k, int def) { return has(k) ? i(k) : def; }
};

const double kDeg = M_PI / 180.;

}  // namespace

double emu_host::vvac_from_pupt_min(const emu_params& p, double pupt_min)
{
    const int nf = p.nflavors;
    double h[9] = {0};
    h[herm_re(nf, 0, 0)] = p.mass1 * p.mass1;
    h[herm_re(nf, 1, 1)] = p.mass2 * p.mass2;
    if (nf == 3) h[herm_re(nf, 2, 2)] = p.mass3 * p.mass3;
    return su_length(nf, h) * emu_host::c4() / pupt_min;
}

extern "C" {

void emu_params_default(emu_params* p)
{
    std::memset(p, 0, sizeof(*p));
    p->nflavors = 2;
    p->shape_order = 2;
    p->precision = EMU_PREC_FP64;
    p->integration_type = 1;
    p->rk_type = 4;
    for (int d = 0; d < 3; d++) { p->ncell[d] = 1; p->nppc[d] = 1; }
    p->nphi_equator = 1;
    p->Lx = p->Ly = p->Lz = 1.0;
    p->max_grid_size = 64;
    p->nsteps = 1;
    p->end_time = 1.0;
    p->write_plot_every = 1;
    p->write_plot_particles_every = 1;
    p->T_in = 10;
    p->Ye_in = 1;
    p->cfl_factor = 0.5;
    p->flavor_cfl_factor = 0.5;
    p->maxError = 1e-6;
    p->direction_generator = 0;
    p->ndirections = 0;
    p->seed = 0;
    p->resort_interval = -1;
    p->fused = 1;
}

int emu_parse_inputs(const char* path, int n_overrides, const char* const* overrides, emu_params* out,
                     char* errbuf, size_t errlen)
{
    auto err = [&](const std::string& m) {
        g_err = m;
        if (errbuf && errlen) {
            std::strncpy(errbuf, m.c_str(), errlen - 1);
            errbuf[errlen - 1] = 0;
        }
        return EMU_ERR_PARSE;
    };
    if (!out) return err("emu_parse_inputs: null output");
    Inputs in;
    if (path) {
        std::ifstream f(path);
        if (!f) return err(std::string("cannot open inputs file ") + path);
        std::string line;
        int ln = 0;
        while (std::getline(f, line)) {
            ln++;
            if (!add_line(in, line)) return err("inputs line " + std::to_string(ln) + ": expected key = value");
        }
    }
    for (int i = 0; i < n_overrides; i++)
        if (!add_line(in, overrides[i])) return err(std::string("bad override: ") + overrides[i]);

    emu_params p;
    emu_params_default(&p);
    Getter g{in, std::string()};
    // extensions (optional)
    p.nflavors = g.i_or("emu.nflavors", 2);
    p.shape_order = g.i_or("emu.shape_order", 2);
    {
        std::string pr = g.has("emu.precision") ? g.str("emu.precision") : std::string("fp64");
        p.precision = (pr == "mixed" || pr == "1") ? EMU_PREC_MIXED : EMU_PREC_FP64;
    }
    p.direction_generator = g.i_or("emu.direction_generator", 0);
    p.ndirections = g.i_or("emu.ndirections", 0);
    p.seed = (uint64_t)g.d_or("emu.seed", 0);
    p.resort_interval = g.i_or("emu.resort_interval", -1);
    p.fused = g.i_or("emu.fused", 1);
    // integrator keys read by the AMReX TimeIntegrator
    p.integration_type = g.i("integration.type");
    if (p.integration_type == 1) p.rk_type = g.i("integration.rk.type");
    // TestParams::Initialize (Parameters.H:52-131); every key is required
    p.simulation_type = g.i("simulation_type");
    g.ivec("ncell", p.ncell);
    p.Lx = g.d("Lx");
    p.Ly = g.d("Ly");
    p.Lz = g.d("Lz");
    g.ivec("nppc", p.nppc);
    p.nphi_equator = g.i("nphi_equator");
    p.max_grid_size = g.i("max_grid_size");
    p.nsteps = g.i("nsteps");
    p.end_time = g.d("end_time");
    p.rho_in = g.d("rho_g_ccm");
    p.Ye_in = g.d("Ye");
    p.T_in = g.d("T_MeV");
    p.cfl_factor = g.d("cfl_factor");
    p.flavor_cfl_factor = g.d("flavor_cfl_factor");
    p.max_adaptive_speedup = g.d("max_adaptive_speedup");
    p.write_plot_every = g.i("write_plot_every");
    p.write_plot_particles_every = g.i("write_plot_particles_every");
    p.do_restart = g.i("do_restart");
    std::string rd = g.str("restart_dir");
    std::strncpy(p.restart_dir, rd.c_str(), sizeof(p.restart_dir) - 1);
    p.maxError = g.d("maxError");
    p.mass1 = g.d("mass1_eV");
    p.mass2 = g.d("mass2_eV");
    p.theta12 = g.d("theta12_degrees");
    p.alpha1 = g.d("alpha1_degrees");
    p.mass1 *= kEV / emu_host::c2();
    p.mass2 *= kEV / emu_host::c2();
    p.theta12 *= kDeg;
    p.alpha1 *= kDeg;
    // NUM_FLAVORS>=2 is always true in the reference: the 3-flavor keys are required (Parameters.H:86-97)
    p.mass3 = g.d("mass3_eV");
    p.theta13 = g.d("theta13_degrees");
    p.theta23 = g.d("theta23_degrees");
    p.alpha2 = g.d("alpha2_degrees");
    p.deltaCP = g.d("deltaCP_degrees");
    p.mass3 *= kEV / emu_host::c2();
    p.theta13 *= kDeg;
    p.theta23 *= kDeg;
    p.alpha2 *= kDeg;
    p.deltaCP *= kDeg;
    if (p.simulation_type == 3) {
        p.st3_amplitude = g.d("st3_amplitude");
        p.st3_wavelength_fraction_of_domain = g.i("st3_wavelength_fraction_of_domain");
    }
    if (p.simulation_type == 4) {
        p.st4_theta = g.d("st4_theta");
        p.st4_thetabar = g.d("st4_thetabar");
        p.st4_phi = g.d("st4_phi");
        p.st4_phibar = g.d("st4_phibar");
        p.st4_ndens = g.d("st4_ndens");
        p.st4_ndensbar = g.d("st4_ndensbar");
        p.st4_fluxfac = g.d("st4_fluxfac");
        p.st4_fluxfacbar = g.d("st4_fluxfacbar");
        p.st4_amplitude = g.d("st4_amplitude");
    }
    if (p.simulation_type == 5) {
        p.st5_nnue = g.d("st5_nnue"); p.st5_nnua = g.d("st5_nnua"); p.st5_nnux = g.d("st5_nnux");
        p.st5_fxnue = g.d("st5_fxnue"); p.st5_fxnua = g.d("st5_fxnua"); p.st5_fxnux = g.d("st5_fxnux");
        p.st5_fynue = g.d("st5_fynue"); p.st5_fynua = g.d("st5_fynua"); p.st5_fynux = g.d("st5_fynux");
        p.st5_fznue = g.d("st5_fznue"); p.st5_fznua = g.d("st5_fznua"); p.st5_fznux = g.d("st5_fznux");
        p.st5_amplitude = g.d("st5_amplitude");
    }
    if (!g.missing.empty()) return err("missing required inputs key: " + g.missing);
    std::string why;
    if (!emu_host::validate(p, why)) return err(why);
    *out = p;
    return EMU_OK;
}


int emu_vvac_max(const emu_params* p, const double* records, int64_t n, double* out)
{
    if (!p || !out || (n > 0 && !records)) return EMU_ERR_ARG;
    const int nf = p->nflavors, nr = 3 + 8 + 2 * (2 + nf * nf);
    double pupt_min = INFINITY;
    for (int64_t i = 0; i < n; i++) pupt_min = std::min(pupt_min, records[i * nr + 3 + 7]);
    *out = emu_host::vvac_from_pupt_min(*p, pupt_min);
    return EMU_OK;
}

int emu_write_plotfile_host(const emu_params* p, const char* dir, double time, int step, const double* mesh,
                            const double* records, int64_t n)
{
    if (!p || !dir || !mesh) return EMU_ERR_ARG;
    std::string why;
    if (!emu_host::write_plotfile(*p, dir, time, step, mesh, records, records ? n : 0, why)) {
        g_err = why;
        return EMU_ERR_IO;
    }
    return EMU_OK;
}

int emu_read_particles(const char* plotfile_dir, int nflavors, double* out, int64_t capacity, int64_t* n_out,
                       double* time, int* step)
{
    if (!plotfile_dir || !n_out) return EMU_ERR_ARG;
    const std::string root(plotfile_dir);
    std::ifstream h(root + "/neutrinos/Header");
    if (!h) { g_err = "cannot open " + root + "/neutrinos/Header"; return EMU_ERR_IO; }
    std::string version;
    int dim = 0, nre = 0, nie = 0, ckpt = 0, finest = 0;
    long long np = 0, nextid = 0;
    h >> version >> dim >> nre;
    std::string nm;
    for (int i = 0; i < nre; i++) h >> nm;
    h >> nie;
    for (int i = 0; i < nie; i++) h >> nm;
    h >> ckpt >> np >> nextid >> finest;
    const int nreal = dim + nre, nint = ckpt ? 2 + nie : 0;
    if (nreal != 3 + 8 + 2 * (2 + nflavors * nflavors)) { g_err = "particle layout does not match nflavors"; return EMU_ERR_IO; }
    std::vector<int> ngrids(finest + 1);
    for (auto& x : ngrids) h >> x;
    *n_out = np;
    if (out) {
        if (capacity < np) return EMU_ERR_ARG;
        long long ip = 0;
        for (int lev = 0; lev <= finest; lev++)
            for (int gi = 0; gi < ngrids[lev]; gi++) {
                long long which, count, where;
                h >> which >> count >> where;
                if (count == 0) continue;
                char fn[64];
                std::snprintf(fn, sizeof fn, "/neutrinos/Level_%d/DATA_%05lld", lev, which);
                std::ifstream d(root + fn, std::ios::binary);
                if (!d) { g_err = std::string("cannot open ") + root + fn; return EMU_ERR_IO; }
                d.seekg(where + (long long)count * nint * 4);
                d.read(reinterpret_cast<char*>(out + ip * nreal), sizeof(double) * count * nreal);
                ip += count;
            }
    }
    // time and step from the mesh plotfile header (PlotFileData, IO.cpp:48-55)
    std::ifstream ph(root + "/Header");
    if (ph && (time || step)) {
        std::string line;
        std::getline(ph, line);
        int ncomp = 0;
        ph >> ncomp;
        for (int i = 0; i < ncomp; i++) ph >> line;
        int sd;
        double t;
        int fl;
        ph >> sd >> t >> fl;
        if (time) *time = t;
        std::getline(ph, line);
        for (int i = 0; i < 4; i++) std::getline(ph, line);   // lo, hi, ref ratio, domain
        int st = 0;
        ph >> st;
        if (step) *step = st;
    }
    return EMU_OK;
}

}  // extern "C"
