// B200 (sm_100a) GFN2-xTB energy + gradient engine behind the C ABI of include/axtb_gpu.h.
//
// Host side: validation and model set-up of every molecule (basis from the STO-nG tables,
// H0/ES/AES/D4/repulsion parameters, electron counts; crates/axtb/src/gfn2.rs:34-133,
// crates/axtb/src/basis.rs:20-229, crates/base/src/molecule.rs:35-99, crates/axtb/src/xtb.rs:1159-1212),
// the flat device layout of a batch, and the SCF driver (crates/axtb/src/scf/driver.rs:180-299,
// crates/axtb/src/xtb.rs:437-861). Device side: the kernels of k_geometry.cuh, k_integrals.cuh,
// k_scf.cuh and team_kernel.cuh. Single translation unit, so every kernel is in this library.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <queue>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/axtb_gpu.h"
#include "common.cuh"
#include "k_geometry.cuh"
#include "k_integrals.cuh"
#include "k_scf.cuh"
#include "k_solvation.cuh"
#include "params/gfn2_tables.h"
#include "team_kernel.cuh"
#include "chase.cuh"

using std::vector;

namespace {

// ------------------------------------------------------------------ constants (crates/base/src/units.rs)
const double PI_ = 3.14159265358979323846;
const double AATOAU = 1.0 / (5.29177210544e-11 * 1e10);
const double KB_HARTREE = 3.1668115634564e-6;
const double MCTC_AATOAU =
    1.0 / ((6.62607015e-34 / (2.0 * PI_)) / (9.1093837015e-31 * 299792458.0 * 7.2973525693e-3) * 1e10);
const double ATOMIC_RAD_AA[86] = {
    0.32, 0.37, 1.30, 0.99, 0.84, 0.75, 0.71, 0.64, 0.60, 0.62, 1.60, 1.40, 1.24, 1.14, 1.09, 1.04, 1.00,
    1.01, 2.00, 1.74, 1.59, 1.48, 1.44, 1.30, 1.29, 1.24, 1.18, 1.17, 1.22, 1.20, 1.23, 1.20, 1.20, 1.18,
    1.17, 1.16, 2.15, 1.90, 1.76, 1.64, 1.56, 1.46, 1.38, 1.36, 1.34, 1.30, 1.36, 1.40, 1.42, 1.40, 1.40,
    1.37, 1.36, 1.36, 2.38, 2.06, 1.94, 1.84, 1.90, 1.88, 1.86, 1.85, 1.83, 1.82, 1.81, 1.80, 1.79, 1.77,
    1.77, 1.78, 1.74, 1.64, 1.58, 1.50, 1.41, 1.36, 1.32, 1.30, 1.30, 1.32, 1.44, 1.45, 1.50, 1.42, 1.48, 1.46};
const double FREQ[23] = {0.000001, 0.050000, 0.100000, 0.200000, 0.300000, 0.400000, 0.500000, 0.600000,
                         0.700000, 0.800000, 0.900000, 1.000000, 1.200000, 1.400000, 1.600000, 1.800000,
                         2.000000, 2.500000, 3.000000, 4.000000, 5.000000, 7.500000, 10.00000};

thread_local std::string g_last_error;

struct Fail : std::runtime_error {
    int code;
    Fail(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CK(x)                                                                                   \
    do {                                                                                        \
        cudaError_t err__ = (x);                                                                \
        if (err__ != cudaSuccess) throw Fail(AXTB_ERR_DEVICE, std::string("CUDA: ") + cudaGetErrorString(err__) + " at " #x); \
    } while (0)

// ------------------------------------------------------------------ host model of one molecule
struct HShell {
    int l, np, z, ish;
    double a[6], c[6], amin;
};

HShell sto_shell(int z, int ish) {
    using namespace gfn2tab;
    int ng = NUMBER_OF_PRIMITIVES[z - 1][ish], n = PRINCIPAL_QUANTUM_NUMBER[z - 1][ish], l = ANG_SHELL[z - 1][ish];
    double zeta = SLATER_EXPONENT[z - 1][ish];
    int ityp = (l == 0 ? n : l == 1 ? 4 + n : 7 + n) - 1;
    HShell s{};
    s.l = l;
    s.np = ng;
    s.z = z;
    s.ish = ish;
    double z2 = zeta * zeta;
    auto fill = [&](const double* a, const double* c) {
        for (int i = 0; i < ng; i++) {
            s.a[i] = a[i] * z2;
            s.c[i] = c[i];
        }
    };
    switch (ng) {
        case 1: s.a[0] = P_ALPHA1[ityp] * z2; s.c[0] = 1.0; break;
        case 2: fill(P_ALPHA2[ityp], P_COEFF2[ityp]); break;
        case 3: fill(P_ALPHA3[ityp], P_COEFF3[ityp]); break;
        case 4: fill(P_ALPHA4[ityp], P_COEFF4[ityp]); break;
        case 5: fill(P_ALPHA5[ityp], P_COEFF5[ityp]); break;
        case 6:
            if (n == 6) fill(l == 0 ? P_ALPHA_6S : P_ALPHA_6P, l == 0 ? P_COEFF_6S : P_COEFF_6P);
            else fill(P_ALPHA6[ityp], P_COEFF6[ityp]);
            break;
        default: throw Fail(AXTB_ERR_INPUT, "STO-NG: unsupported primitive count");
    }
    const double DF[3] = {1.0, 1.0, 3.0};
    s.amin = INFINITY;
    for (int i = 0; i < ng; i++) {
        double r = std::sqrt(4.0 * s.a[i]), pw = 1.0;
        for (int k = 0; k < l; k++) pw *= r;
        s.c[i] *= std::pow(2.0 / PI_ * s.a[i], 0.75) * pw / std::sqrt(DF[l]);
        s.amin = std::min(s.amin, s.a[i]);
    }
    return s;
}

double rcov_codata(int z) { return 4.0 / 3.0 * (gfn2tab::COVALENT_RAD_2009_AA[z - 1] * AATOAU); }
double rcov_mctc(int z) { return 4.0 / 3.0 * (MCTC_AATOAU * gfn2tab::COVALENT_RAD_2009_AA[z - 1]); }

// ------------------------------------------------------------------ conventions
// The settings that differ between axtb's default conventions, the xtb 6.8.0 program's and
// tblite 0.8.0's (crates/axtb/src/conventions.rs:150-353 ConventionParams): Boltzmann constant
// and aufbau limit, EEQ start and its CN, element tables, real-space cutoffs, integral
// screening, default mixer and the potentials of the gradient. Not carried over: the per-triple
// ATM order and the full eigensolver of the program conventions (the same numbers up to
// round-off as the pair sums and occupied-only solve used for all three), and the xtb 6.7.1 row.
const double KB_XTB_TBLITE = 3.166808578545117e-06;  // crates/base/src/units.rs:81
struct Conv {
    int id = 0;  // 0 axtb, 1 xtb (6.8.0), 2 tblite (0.8.0)
    double kb = KB_HARTREE, aufbau_max_etemp = 0.0;
    bool eeq_guess = true;
    double eeq_cn_cut = 25.0, eeq_cap = 8.0;
    double cn_cut = 40.0, rep_cut = 40.0, d4_cn_cut = 40.0, d2_cut = 72.0, d2_w = 1.0, d3_cut = 40.0, d3_w = 1.0;
    bool output_aes = false;
    int default_mixer = 0;  // 0 auto, 1 Broyden
    explicit Conv(int c) : id(c) {
        if (c == 0) return;
        kb = KB_XTB_TBLITE;
        cn_cut = rep_cut = 25.0;
        d4_cn_cut = 30.0;  // RealspaceCutoff::TBLITE_GFN2 (crates/d4/src/disp.rs:44-47)
        d2_cut = 50.0;
        d3_cut = 25.0;
        d2_w = d3_w = 0.05;
        default_mixer = 1;
        if (c == 1) {
            aufbau_max_etemp = 0.1;
            eeq_cn_cut = 40.0;  // the xtb program's guess CN: its D4 radii, 40 bohr, no cap
            eeq_cap = 0.0;
            output_aes = true;
        } else {
            eeq_guess = false;
        }
    }
    double en(int z) const { return id == 1 ? gfn2tab::XTB_PAULING_EN[z - 1] : gfn2tab::PAULING_EN[z - 1]; }
    double atomic_rad(int z) const {
        return id == 1 ? gfn2tab::XTB_ATOMIC_RAD[z - 1]
                       : id == 2 ? MCTC_AATOAU * ATOMIC_RAD_AA[z - 1] : ATOMIC_RAD_AA[z - 1] * AATOAU;
    }
    double cn_rcov(int z) const {
        return id == 1 ? gfn2tab::XTB_COVALENT_RAD_D3[z - 1] : id == 2 ? rcov_mctc(z) : rcov_codata(z);
    }
    double d4_rcov(int z) const { return id == 1 ? gfn2tab::XTB_D4_RCOV[z - 1] : id == 2 ? rcov_mctc(z) : rcov_codata(z); }
    double d4_en(int z) const { return id == 1 ? gfn2tab::XTB_D4_EN[z - 1] : gfn2tab::PAULING_EN[z - 1]; }
    double eeq_rcov(int z) const { return id == 1 ? gfn2tab::XTB_D4_RCOV[z - 1] : rcov_mctc(z); }
    // primitive screening (crates/axtb/src/gfn2.rs:58-62, crates/axtb/src/basis.rs:135-143)
    static double tblite_cut(double acc) {
        acc = std::min(std::max(acc, 1.0e-4), 1.0e3);
        return std::min(std::max(25.0 - 10.0 * std::log10(acc), 5.0), 25.0);
    }
    double intcut(double acc) const {
        return id == 0 ? std::max(25.0 - 10.0 * std::log10(acc), 20.0) : id == 1 ? tblite_cut(acc) : tblite_cut(1.0);
    }
    // tblite's atom-pair cutoff of the integrals, squared (crates/axtb/src/basis.rs:247-249)
    double pair_cut2(double acc, double min_alpha) const {
        if (id != 2) return INFINITY;
        double pc = std::min(std::sqrt(2.0 * tblite_cut(acc) / min_alpha), 40.0);
        return pc * pc;
    }
};

struct HostMol {
    int nat = 0;
    vector<int> Z;
    vector<double> xyz;
    double charge = 0.0;
    int uhf = -1;
    double nalpha = 0, nbeta = 0;
    int nsh = 0, nao = 0;
};

// validation (crates/base/src/molecule.rs:35-99) and electrons (crates/axtb/src/xtb.rs:1178-1212)
void check_molecule(HostMol& m) {
    using namespace gfn2tab;
    if (m.nat <= 0) throw Fail(AXTB_ERR_INPUT, "molecule has no atoms");
    for (int z : m.Z) {
        if (z <= 0 || z > 118) throw Fail(AXTB_ERR_INPUT, "invalid atomic number " + std::to_string(z));
        if (z > 86) throw Fail(AXTB_ERR_UNSUPPORTED_ELEMENT, "GFN2-xTB: unsupported element Z=" + std::to_string(z));
    }
    if (!std::isfinite(m.charge)) throw Fail(AXTB_ERR_INPUT, "the charge must be a finite number");
    for (double v : m.xyz)
        if (!std::isfinite(v)) throw Fail(AXTB_ERR_INPUT, "a position is not finite");
    vector<int> ord(m.nat);
    std::iota(ord.begin(), ord.end(), 0);
    std::sort(ord.begin(), ord.end(), [&](int a, int b) { return m.xyz[3 * a] < m.xyz[3 * b]; });
    for (int k = 0; k < m.nat; k++)
        for (int q = k + 1; q < m.nat; q++) {
            int i = ord[k], j = ord[q];
            if (m.xyz[3 * j] - m.xyz[3 * i] >= 0.1) break;
            double d2 = 0;
            for (int c = 0; c < 3; c++) d2 += (m.xyz[3 * i + c] - m.xyz[3 * j + c]) * (m.xyz[3 * i + c] - m.xyz[3 * j + c]);
            if (std::sqrt(d2) < 0.1)
                throw Fail(AXTB_ERR_INPUT, "atoms " + std::to_string(std::min(i, j) + 1) + " and " +
                                               std::to_string(std::max(i, j) + 1) + " are closer than 0.1 bohr");
        }
    if (m.charge != std::floor(m.charge)) throw Fail(AXTB_ERR_INPUT, "the charge must be an integer");
    double nref = 0.0;
    m.nsh = m.nao = 0;
    for (int z : m.Z)
        for (int ish = 0; ish < NSHELL[z - 1]; ish++) {
            nref += REFERENCE_OCC[z - 1][ANG_SHELL[z - 1][ish]];
            m.nsh++;
            m.nao += 2 * ANG_SHELL[z - 1][ish] + 1;
        }
    double nocc = nref - m.charge;
    long nel = std::lround(nocc);
    long par = ((nel % 2) + 2) % 2;
    long nuhf = par;
    if (m.uhf >= 0) {
        if ((m.uhf % 2) != par) throw Fail(AXTB_ERR_INPUT, "electron count and unpaired electrons are not compatible");
        nuhf = m.uhf;
    }
    if (nocc < 0.0) throw Fail(AXTB_ERR_INPUT, "the charge leaves a negative electron count");
    if (nuhf > nocc) throw Fail(AXTB_ERR_INPUT, "more unpaired electrons than electrons");
    m.nalpha = (nocc + nuhf) / 2.0;
    m.nbeta = (nocc - nuhf) / 2.0;
    if (m.nalpha > m.nao + 1e-9) throw Fail(AXTB_ERR_INPUT, "too many electrons for the basis");
}

struct Opt {
    double acc = 1.0, etemp = 300.0, damping = 0.4;
    int max_iter = 250, guess = 0, precision = 0, device = 0;
    int mixer = -1;  // -1 the conventions' mixer, 0 auto (Broyden, then DIIS from the start), 1 Broyden, 2 DIIS
    int conventions = 0;  // 0 axtb, 1 xtb (6.8.0), 2 tblite (0.8.0)
    int solv = -1;        // implicit solvation: -1 none, 0 ALPB, 1 GBSA
    std::string solvent;  // its solvent (xtb's names and aliases)
    int solv_state = 0;   // reference state: 0 gsolv, 1 bar1M, 2 reference
    int dispersion = 1;   // 0: leave the D4 term out (crates/axtb/src/lib.rs:107, 185-187)
    int band_max_nao = -1;  // schedule: two-stage reduction below this many AOs (-1: default)
    int grid_min_nao = -1;  // schedule: whole-grid teams from this many AOs (-1: default)
};

// default schedule of the dense algebra (axtb_b200.autotune measures both crossovers on a device):
// the two-stage reduction below 64 AOs (measured on B200: per molecule it is also cheaper between
// 224 and 416 AOs with the bulge chasing on chip, but whole batches run no faster, the eigen phase
// then being three launches with three tails)
constexpr int DEFAULT_BAND_MAX_NAO = 64;
constexpr int STATIC_BAND_MAX_NAO = 64;
constexpr int DEFAULT_GRID_MIN_NAO = 1024;

// ------------------------------------------------------------------ solvation parameters
// the parameter set of a solvent name (crates/solvation/src/lib.rs:255-272: trimmed, lower case,
// xtb's aliases, the model's table); nullptr when the model has none
const solvtab::SolventParam* solvent_param(const std::string& name, bool alpb) {
    using namespace solvtab;
    size_t a = name.find_first_not_of(" \t\n"), b = name.find_last_not_of(" \t\n");
    std::string s = a == std::string::npos ? std::string() : name.substr(a, b - a + 1);
    for (char& c : s) c = (char)std::tolower((unsigned char)c);
    for (const auto& al : ALIASES)
        if (s == al.alias) {
            s = al.name;
            break;
        }
    if (alpb) {
        for (const auto& t : ALPB_SOLVENTS)
            if (s == t.name) return &PARAMS[t.param];
    } else {
        for (const auto& t : GBSA_SOLVENTS)
            if (s == t.name) return &PARAMS[t.param];
    }
    return nullptr;
}

void check_options(const Opt& o) {
    if (!(o.acc > 0.0 && std::isfinite(o.acc))) throw Fail(AXTB_ERR_INPUT, "SCF accuracy must be a positive number");
    if (!(o.etemp >= 0.0 && std::isfinite(o.etemp))) throw Fail(AXTB_ERR_INPUT, "electronic temperature must be >= 0 K");
    if (!(o.damping > 0.0 && o.damping <= 1.0)) throw Fail(AXTB_ERR_INPUT, "SCF damping must be in (0, 1]");
    if (o.max_iter <= 0) throw Fail(AXTB_ERR_INPUT, "the SCF needs at least 1 iteration");
    if (o.precision != 0 && o.precision != 1) throw Fail(AXTB_ERR_INPUT, "precision must be 0 (FP64) or 1 (split)");
    if (o.mixer < -1 || o.mixer > 2) throw Fail(AXTB_ERR_INPUT, "unknown SCF mixer (0 auto, 1 Broyden, 2 DIIS)");
    if (o.conventions < 0 || o.conventions > 2) throw Fail(AXTB_ERR_INPUT, "unknown conventions (0 axtb, 1 xtb, 2 tblite)");
    if (o.solv < -1 || o.solv > 1) throw Fail(AXTB_ERR_INPUT, "unknown solvation model (-1 none, 0 ALPB, 1 GBSA)");
    if (o.solv >= 0 && (o.solv_state < 0 || o.solv_state > 2))
        throw Fail(AXTB_ERR_INPUT, "unknown solvation reference state (0 gsolv, 1 bar1M, 2 reference)");
    if (o.solv >= 0 && !solvent_param(o.solvent, o.solv == 0))
        throw Fail(AXTB_ERR_INPUT, "solvation: unknown solvent '" + o.solvent + "' for this model");
}

// ------------------------------------------------------------------ device arena
struct Arena {
    char* base = nullptr;
    size_t size = 0, used = 0;
    template <class T>
    T* take(size_t n) {
        size_t bytes = ((n * sizeof(T)) + 255) & ~size_t(255);
        if (used + bytes > size) throw Fail(AXTB_ERR_DEVICE, "device arena exhausted");
        T* p = reinterpret_cast<T*>(base + used);
        used += bytes;
        return p;
    }
};

template <class T>
size_t padded(size_t n) {
    return ((n * sizeof(T)) + 255) & ~size_t(255);
}

}  // namespace

// ------------------------------------------------------------------ the batch engine
struct Moments;  // a molecule's SCC moments (capi.cuh)
struct AxtbBatch {
    int device = 0;
    cudaStream_t st = nullptr;
    Opt opt;
    vector<HostMol> mols;
    int nmol = 0, natT = 0, nshT = 0, naoT = 0;
    long long nnT = 0, npairT = 0, npdT = 0, nvecT = 0, nsqT = 0, ntiles = 0, nwk = 0, nhist = 0, ngamT = 0;
    int hist_cap = 0, nsp = 0;
    int mixer_kind = 0;      // the mixer plan of the run: 0 auto, 1 Broyden, 2 DIIS
    bool restart = false;    // molecules start from their previous converged moments
    bool retry_fresh = true; // ... and one that then ends unconverged runs once more from the guess
    bool eeq_guess = true;   // the conventions start from EEQ charges
    axg::Batch B{};
    axg::State S{};
    axg::TeamPlan P{};
    axg::ChasePlan CP{};    // molecules whose band k_chase reduces (stage 2 on chip)
    int nchase = 0, chase_grid = 0;
    void* dmem = nullptr;
    void* hpin = nullptr;  // pinned staging
    size_t hpin_size = 0;
    long long *d_pair0 = nullptr, *d_pd0 = nullptr, *d_tile0 = nullptr, *d_sq0 = nullptr;
    double *d_wt = nullptr, *d_tt = nullptr, *d_eatm = nullptr;
    int grid = 0;
    int64_t launches = 0;
    // host copies of the per-molecule offsets
    vector<long long> m_mat0, m_pair0, m_vec0;
    vector<int> m_at0, m_sh0, m_ao0;
    vector<double> e_rep, e_atm;
    std::string err;

    void build(const vector<HostMol>& in, const Opt& o);
    // want_levels: every orbital energy of the result (the SCF itself needs the lowest ones only)
    void run(bool want_grad, bool warm = false, bool want_levels = false);
    cudaEvent_t phase_ev[4] = {nullptr, nullptr, nullptr, nullptr};  // start, SCF start, SCF end, end
    vector<int> h_warm;     // per molecule: the last run's result started from previous or given moments
    // profiling and traffic accounting
    struct Rec {
        const char* name;
        cudaEvent_t e0, e1;
        double flops, bytes;
    };
    struct Acc {
        long long launches = 0;
        double ms = 0, flops = 0, bytes = 0;
    };
    bool profiling = false;
    double team_cycles[axg::TEAM_CYCLE_SLOTS] = {0};
    std::vector<double> eigen_ms;  // each eigen launch of the last profiled run (ms)
    vector<Rec> recs;
    std::map<std::string, Acc> prof;
    int* h_act = nullptr;          // pinned copy of the active flags
    double* h_stage = nullptr;     // pinned staging for positions and results
    size_t h_stage_len = 0;
    long long h2d_bytes = 0, d2h_bytes = 0;
    void begin_launch(const char* name, double flops, double bytes);
    void end_launch();
    void resolve_profile();
    void extract(AxtbResult* outs, int32_t* status, bool want_grad);
    void upload_positions(const double* host_xyz, bool device_ptr);
    void put_moments(int m, const Moments& w);
    Moments get_moments(int m);
    ~AxtbBatch();
};

AxtbBatch::~AxtbBatch() {
    for (auto& e : phase_ev)
        if (e) cudaEventDestroy(e);
    if (h_act) cudaFreeHost(h_act);
    if (h_stage) cudaFreeHost(h_stage);
    if (dmem) cudaFree(dmem);
    if (hpin) cudaFreeHost(hpin);
    if (st) cudaStreamDestroy(st);
}

void AxtbBatch::build(const vector<HostMol>& in, const Opt& o) {
    using namespace gfn2tab;
    opt = o;
    mols = in;
    nmol = (int)mols.size();
    if (nmol <= 0) throw Fail(AXTB_ERR_INPUT, "empty batch");
    const Conv cv(o.conventions);
    mixer_kind = o.mixer < 0 ? cv.default_mixer : o.mixer;
    eeq_guess = cv.eeq_guess;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0)
        throw Fail(AXTB_ERR_DEVICE, "no CUDA device: the GFN2-xTB engine has no CPU path");
    device = o.device;
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    for (auto& e : phase_ev) CK(cudaEventCreate(&e));
    // ---- host layout
    vector<int> m_nat(nmol), m_nsh(nmol), m_nao(nmol), m_dim(nmol);
    vector<long long> m_hist0(nmol), m_pd0(nmol), m_tile0(nmol), m_wk0(nmol), m_sq0(nmol), m_gam0(nmol);
    vector<double> m_na(nmol), m_nb(nmol), m_ch(nmol);
    m_at0.resize(nmol);
    m_sh0.resize(nmol);
    m_ao0.resize(nmol);
    m_mat0.resize(nmol);
    m_pair0.resize(nmol);
    m_vec0.resize(nmol);
    // Broyden keeps max_iter history vectors (its memory, crates/axtb/src/xtb.rs:598) up to
    // BROYDEN_MAX_HIST when the histories of the whole batch fit in 1 GiB, else 64 (a molecule
    // that needs more ends its Broyden attempt there); the span of each molecule also holds the
    // DIIS history
    {
        long long vec = 0;
        for (auto& h : mols) vec += h.nsh + 9LL * h.nat;
        int full = std::min(o.max_iter, axg::BROYDEN_MAX_HIST);
        double bytes = 16.0 * full * (double)vec + 16.0 * nmol * (double)full * full;  // df, u; a and beta
        hist_cap = bytes <= (double)(1LL << 30) ? full : std::min(o.max_iter, 64);
    }
    const int hist_span = std::max(hist_cap, axg::DIIS_SLOTS);
    natT = nshT = naoT = 0;
    nnT = npairT = npdT = nvecT = nsqT = ntiles = nwk = nhist = ngamT = 0;
    for (int m = 0; m < nmol; m++) {
        HostMol& h = mols[m];
        m_nat[m] = h.nat;
        m_nsh[m] = h.nsh;
        m_nao[m] = h.nao;
        m_dim[m] = h.nsh + 9 * h.nat;
        m_at0[m] = natT;
        m_sh0[m] = nshT;
        m_ao0[m] = naoT;
        m_mat0[m] = nnT;
        m_pair0[m] = npairT;
        m_pd0[m] = npdT;
        m_vec0[m] = nvecT;
        m_hist0[m] = nhist;
        m_sq0[m] = nsqT;
        m_gam0[m] = ngamT;
        m_tile0[m] = ntiles;
        m_wk0[m] = nwk;
        m_na[m] = h.nalpha;
        m_nb[m] = h.nbeta;
        m_ch[m] = h.charge;
        long long n = h.nao;
        natT += h.nat;
        nshT += h.nsh;
        naoT += h.nao;
        nnT += (std::max(n * n, 64LL * 64LL) + 31) & ~31LL;  // 256-byte aligned planes
        npairT += (long long)h.nat * (h.nat - 1) / 2;
        npdT += (long long)h.nat * (h.nat + 1) / 2;
        nvecT += m_dim[m];
        nhist += (long long)hist_span * m_dim[m];
        nsqT += (long long)h.nat * h.nat;
        ngamT += (long long)h.nsh * h.nsh;
        long long nt = (n + 31) / 32;
        ntiles += nt * (nt + 1) / 2;  // Fock tile pairs (I >= J)
        long long nw = std::max(n, 64LL);
        nwk += (axg::team_workspace((int)n) + 31) & ~31LL;
    }
    // atoms / shells / AOs
    vector<int> a_Z(natT), a_mol(natT), a_sh0(natT), a_nsh(natT), a_ao0(natT), a_sp(natT);
    vector<double> a_rcov(natT), a_rad(natT), a_amin(natT), a_rcov_eeq(natT), a_en(natT), a_aes_rad(natT),
        a_aes_vcn(natT), a_dk(natT), a_qk(natT), a_ra(natT), a_rz(natT), a_chi(natT), a_eta(natT), a_kcn(natT),
        a_erad(natT);
    vector<int> s_l(nshT), s_np(nshT), s_at(nshT), s_ao0(nshT), s_ish(nshT), s_mol(nshT), s_Z(nshT);
    vector<double> s_alpha((size_t)nshT * 6, 0.0), s_coeff((size_t)nshT * 6, 0.0), s_amin(nshT), s_se0(nshT),
        s_kcn(nshT), s_shpoly(nshT), s_refocc(nshT), s_hard(nshT), s_gam3(nshT), s_slater(nshT);
    vector<int> o_sh(naoT), o_at(naoT);
    vector<int> species;
    const double SHD[3] = {1.0, 0.5, 0.25};
    {
        int ia = 0, is = 0, io = 0;
        for (int m = 0; m < nmol; m++) {
            const HostMol& h = mols[m];
            for (int i = 0; i < h.nat; i++, ia++) {
                int z = h.Z[i];
                auto it = std::find(species.begin(), species.end(), z);
                int sp = (int)(it - species.begin());
                if (it == species.end()) species.push_back(z);
                a_Z[ia] = z;
                a_mol[ia] = m;
                a_sh0[ia] = is;
                a_nsh[ia] = NSHELL[z - 1];
                a_ao0[ia] = io;
                a_sp[ia] = sp;
                a_rcov[ia] = cv.cn_rcov(z);
                a_rad[ia] = cv.atomic_rad(z);
                a_rcov_eeq[ia] = cv.eeq_rcov(z);
                a_en[ia] = cv.en(z);
                a_aes_rad[ia] = P_RAD[z - 1];
                a_aes_vcn[ia] = P_VCN[z - 1];
                a_dk[ia] = P_DKERNEL[z - 1];
                a_qk[ia] = P_QKERNEL[z - 1];
                a_ra[ia] = REP_ALPHA[z - 1];
                a_rz[ia] = REP_ZEFF[z - 1];
                if (z > 103) throw Fail(AXTB_ERR_UNSUPPORTED_ELEMENT, "EEQ: unsupported element");
                a_chi[ia] = EEQ_CHI[z - 1];
                a_eta[ia] = EEQ_ETA[z - 1];
                a_kcn[ia] = EEQ_KCNCHI[z - 1];
                a_erad[ia] = EEQ_RAD[z - 1];
                double amin = INFINITY;
                for (int ish = 0; ish < NSHELL[z - 1]; ish++, is++) {
                    HShell sh = sto_shell(z, ish);
                    int l = sh.l;
                    s_l[is] = l;
                    s_np[is] = sh.np;
                    s_at[is] = ia;
                    s_ao0[is] = io;
                    s_ish[is] = ish;
                    s_mol[is] = m;
                    s_Z[is] = z;
                    for (int p = 0; p < 6; p++) {
                        s_alpha[(size_t)is * 6 + p] = sh.a[p];
                        s_coeff[(size_t)is * 6 + p] = sh.c[p];
                    }
                    s_amin[is] = sh.amin;
                    amin = std::min(amin, sh.amin);
                    s_se0[is] = P_SELFENERGY[z - 1][ish];
                    s_kcn[is] = P_KCN[z - 1][l];
                    s_shpoly[is] = P_SHPOLY[z - 1][l];
                    s_refocc[is] = REFERENCE_OCC[z - 1][l];
                    s_hard[is] = HUBBARD_PARAMETER[z - 1] * SHELL_HUBBARD[z - 1][l];
                    s_gam3[is] = P_HUBBARD_DERIVS[z - 1] * SHD[l];
                    s_slater[is] = SLATER_EXPONENT[z - 1][ish];
                    for (int k = 0; k < 2 * l + 1; k++, io++) {
                        o_sh[io] = is;
                        o_at[io] = ia;
                    }
                }
                a_amin[ia] = amin;
            }
        }
    }
    // D4 species tables (crates/d4/src/model.rs:140-217, 319-386)
    nsp = (int)species.size();
    vector<int> sp_nref(nsp), sp_ngw((size_t)nsp * 7, 1);
    vector<double> sp_refcn((size_t)nsp * 7, 0.0), sp_refq((size_t)nsp * 7, 0.0), sp_zeff(nsp), sp_gi(nsp),
        sp_rcov(nsp), sp_en(nsp), sp_rr((size_t)nsp * nsp), sp_r0((size_t)nsp * nsp);
    vector<double> aiw((size_t)nsp * 7 * 23, 0.0), c6ref((size_t)nsp * nsp * 49, 0.0), r4r2(nsp);
    for (int sp = 0; sp < nsp; sp++) {
        int z = species[sp], nr = REFN[z - 1];
        sp_nref[sp] = nr;
        int cnc[20] = {0};
        cnc[0] = 1;
        auto icn = [](double x) { long v = std::lround(x); return (int)std::min(19L, std::max(0L, v)); };
        for (int r = 0; r < nr; r++) cnc[icn(REFCN[z - 1][r])]++;
        for (int r = 0; r < nr; r++) {
            int c = cnc[icn(REFCN[z - 1][r])];
            sp_ngw[sp * 7 + r] = c * (c + 1) / 2;
            sp_refcn[sp * 7 + r] = REFCOVCN[z - 1][r];
            sp_refq[sp * 7 + r] = REFQ_GFN2[z - 1][r];
        }
        sp_zeff[sp] = EFFECTIVE_NUCLEAR_CHARGE[z - 1];
        sp_gi[sp] = CHEMICAL_HARDNESS[z - 1] * 2.0;
        sp_rcov[sp] = cv.d4_rcov(z);
        sp_en[sp] = cv.d4_en(z);
        r4r2[sp] = std::sqrt(0.5 * (R4_OVER_R2[z - 1] * std::sqrt((double)z)));
        for (int ir = 0; ir < nr; ir++) {
            int s2 = REFSYS[z - 1][ir];
            if (s2 == 0) continue;
            double iz = EFFECTIVE_NUCLEAR_CHARGE[s2 - 1], gam = CHEMICAL_HARDNESS[s2 - 1] * 2.0;
            double qmod = REFH_GFN2[z - 1][ir] + iz;
            double zv = qmod < 0.0 ? std::exp(3.0) : std::exp(3.0 * (1.0 - std::exp(gam * (1.0 - iz / qmod))));
            for (int k = 0; k < 23; k++) {
                double a = SSCALE[s2 - 1] * SECAIW[s2 - 1][k] * zv;
                double v = ASCALE[z - 1][ir] * (ALPHAIW[z - 1][ir][k] - HCOUNT[z - 1][ir] * a);
                aiw[((size_t)sp * 7 + ir) * 23 + k] = v > 0.0 ? v : 0.0;
            }
        }
    }
    double tw[23];
    tw[0] = 0.5 * (FREQ[1] - FREQ[0]);
    for (int k = 1; k < 22; k++) tw[k] = 0.5 * ((FREQ[k] - FREQ[k - 1]) + (FREQ[k + 1] - FREQ[k]));
    tw[22] = 0.5 * (FREQ[22] - FREQ[21]);
    for (int a = 0; a < nsp; a++)
        for (int b = 0; b <= a; b++)
            for (int r = 0; r < sp_nref[a]; r++)
                for (int s = 0; s < sp_nref[b]; s++) {
                    double acc = 0.0;
                    for (int k = 0; k < 23; k++) acc += aiw[((size_t)a * 7 + r) * 23 + k] * aiw[((size_t)b * 7 + s) * 23 + k] * tw[k];
                    double c6 = 3.0 / PI_ * acc;
                    c6ref[((size_t)(a * nsp + b)) * 49 + r * 7 + s] = c6;
                    c6ref[((size_t)(b * nsp + a)) * 49 + s * 7 + r] = c6;
                }
    for (int a = 0; a < nsp; a++)
        for (int b = 0; b < nsp; b++) {
            double v = 3.0 * r4r2[a] * r4r2[b];
            sp_rr[a * nsp + b] = v;
            sp_r0[a * nsp + b] = 0.52 * std::sqrt(v) + 5.0;
        }
    // one-CTA molecules of 34 AOs up to below band_max_nao reduce to tridiagonal form in two
    // stages, the others (and the whole-grid molecules) in one (AXTB_EIGEN_ONESTAGE=1: all in one stage)
    int band_max = o.band_max_nao >= 0 ? o.band_max_nao : DEFAULT_BAND_MAX_NAO;
    if (std::getenv("AXTB_EIGEN_ONESTAGE")) band_max = 0;
    // stage 2 of those in shared memory (k_chase: one CTA per SM, a cluster pair above CHASE_ROWS
    // AOs) when the device offers the shared memory and clusters (AXTB_STAGE2_IN_TEAM=1: in the
    // team kernel, the band in global memory; the same results)
    int chase_max = 0;
    {
        int optin = 0, clusters = 0;
        CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
        CK(cudaDeviceGetAttribute(&clusters, cudaDevAttrClusterLaunch, device));
        if (optin >= axg::CHASE_DYN_BYTES + axg::CHASE_STATIC_BYTES && clusters &&
            !std::getenv("AXTB_STAGE2_IN_TEAM")) {
            CK(cudaFuncSetAttribute((const void*)axg::k_chase, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    axg::CHASE_DYN_BYTES));
            chase_max = axg::CHASE_MAX_NAO;
        }
    }
    // ---- team plan: molecules from 1024 AOs on run on the whole grid, the rest one per CTA
    int nsm = 0;
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    int per = 0;
    CK(cudaFuncSetAttribute((const void*)axg::k_team, cudaFuncAttributeMaxDynamicSharedMemorySize, axg::SMEM_WORK_BYTES));
    CK(cudaFuncSetAttribute((const void*)axg::k_team_grid, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            axg::SMEM_WORK_BYTES));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, axg::k_team, axg::TEAM_THREADS, axg::SMEM_WORK_BYTES));
    {
        int per_grid = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_grid, axg::k_team_grid, axg::TEAM_THREADS,
                                                         axg::SMEM_WORK_BYTES));
        per = std::min(per, per_grid);
    }
    if (per <= 0) throw Fail(AXTB_ERR_DEVICE, "team kernel does not fit on a multiprocessor");
    grid = nsm * std::min(per, 2);
    vector<int> big, small_off(grid + 1, 0), small_list, head_off, head_list, tail_off, tail_list;
    {
        vector<std::pair<double, int>> smalls, heads, tails;
        // molecules from this many AOs on take the whole grid (AXTB_TEAM_BIG_NAO overrides, e.g.
        // to run small molecules through the grid-wide path in tests)
        int big_nao = o.grid_min_nao > 0 ? o.grid_min_nao : DEFAULT_GRID_MIN_NAO;
        if (const char* e = std::getenv("AXTB_TEAM_BIG_NAO")) big_nao = std::max(1, std::atoi(e));
        // the eigen phase of a molecule whose bulge chasing runs on chip is split over two team
        // launches (before and after k_chase), each balanced on its own: measured shares of a
        // two-stage eigen phase, ~0.2 before (F' and stage 1) and ~0.55 after
        for (int m = 0; m < nmol; m++) {
            int n = m_nao[m];
            if (n >= big_nao) {
                big.push_back(m);
                continue;
            }
            double c = std::pow((double)n + 32.0, 3.0);
            bool chased = n > axg::BW + 1 && n < band_max && n <= chase_max;
            smalls.push_back({c, m});
            heads.push_back({chased ? 0.2 * c : c, m});
            if (chased) tails.push_back({0.55 * c, m});
        }
        // longest first onto the least loaded CTA
        auto lpt = [&](vector<std::pair<double, int>>& items, vector<int>& off, vector<int>& list) {
            std::sort(items.begin(), items.end(), [](auto& x, auto& y) { return x.first > y.first; });
            vector<vector<int>> lists(grid);
            std::priority_queue<std::pair<double, int>, vector<std::pair<double, int>>, std::greater<>> pq;
            for (int g = 0; g < grid; g++) pq.push({0.0, g});
            for (auto& it : items) {
                auto top = pq.top();
                pq.pop();
                lists[top.second].push_back(it.second);
                pq.push({top.first + it.first, top.second});
            }
            off.assign(grid + 1, 0);
            list.clear();
            for (int g = 0; g < grid; g++) {
                off[g + 1] = off[g] + (int)lists[g].size();
                for (int m : lists[g]) list.push_back(m);
            }
        };
        lpt(smalls, small_off, small_list);
        lpt(heads, head_off, head_list);
        lpt(tails, tail_off, tail_list);
    }
    // ---- device allocation (one arena)
    size_t bytes = 0;
    auto addI = [&](size_t n) { bytes += padded<int>(n); };
    auto addD = [&](size_t n) { bytes += padded<double>(n); };
    auto addL = [&](size_t n) { bytes += padded<long long>(n); };
    addI(nmol * 7);
    addL(nmol * 10);
    addL(nmol);                                    // shell gamma matrix offsets
    addD((size_t)std::max(ngamT, 1LL));           // shell gamma matrices
    addD(nmol * 3);
    addD(nmol);  // per-molecule pair cutoffs
    addI(natT * 6);
    addD(natT * 15);
    addI(nshT * 7);
    addD((size_t)nshT * 12 + (size_t)nshT * 9);
    addI(naoT * 2);
    addI(nsp + nsp * 7);
    addD(nsp * 7 * 2 + nsp * 4 + (size_t)nsp * nsp * 49 + (size_t)nsp * nsp * 2);
    addI(big.size() + 1 + small_off.size() + small_list.size() + 1);
    addI(head_off.size());  // the eigen phase's own plans (before and after k_chase)
    addI(head_list.size() + 1);
    addI(tail_off.size());
    addI(tail_list.size() + 1);
    {  // the chase plan (k_chase): offsets per cluster and per CTA, molecule lists
        size_t ncl = (size_t)std::max(1, nsm / 2);
        addI(ncl + 1);
        addI((size_t)nmol + 1);
        addI(2 * ncl + 1);
        addI((size_t)nmol + 1);
    }
    // state
    addD(natT * 3 + natT * 6 + nshT * 2);
    addD((size_t)nnT * 22);
    bytes += padded<unsigned char>((size_t)nnT);
    addD((size_t)naoT * 6);
    addD((size_t)nmol * 2);  // Fermi levels
    addI(nmol * 7);
    addI(nmol);
    addI(nmol);
    addI(nmol);
    addI(nmol);
    addD((size_t)nmol * 8);                          // DIIS scalars
    addD((size_t)nshT + (size_t)natT * 10);          // start moments
    addD((size_t)nshT * 3 + (size_t)natT * 2 + (size_t)natT * 6 + (size_t)natT * 12 + (size_t)nshT + natT * 10);
    addD((size_t)natT * 14);
    addD((size_t)naoT * 11);
    addD((size_t)nvecT * 4 + (size_t)nhist * 2 + (size_t)nmol * hist_cap * hist_cap * 2 + (size_t)nmol * hist_cap);
    addD((size_t)nmol * 14);
    addD((size_t)nmol);  // per-molecule eigen cycles
    addD((size_t)natT * 5 + (size_t)std::max(npairT, 1LL) * 5 + natT + natT * 5);
    addD((size_t)grid * 64 + 64);
    addD((size_t)nsqT * 3 + natT * 2);
    addD((size_t)nwk);
    addL(nmol * 5);
    addD((size_t)nsqT * 2);
    if (o.solv >= 0) {  // solvation: 9 per-atom parameter arrays, 7 per-atom state arrays, lists
        addD((size_t)natT * 9 + nmol);
        addD((size_t)natT * 10 + nmol * 2);
        addI((size_t)natT * axg::SOLV_MAXNB + natT);
    }
    bytes += 1 << 20;
    CK(cudaMalloc(&dmem, bytes));
    Arena ar{(char*)dmem, bytes, 0};
    auto upI = [&](const vector<int>& v) {
        int* p = ar.take<int>(std::max<size_t>(v.size(), 1));
        if (!v.empty()) CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        return (const int*)p;
    };
    auto upD = [&](const vector<double>& v) {
        double* p = ar.take<double>(std::max<size_t>(v.size(), 1));
        if (!v.empty()) CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        return (const double*)p;
    };
    auto upL = [&](const vector<long long>& v) {
        long long* p = ar.take<long long>(std::max<size_t>(v.size(), 1));
        if (!v.empty()) CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(long long), cudaMemcpyHostToDevice, st));
        return p;
    };
    axg::Batch& b = B;
    b.nmol = nmol;
    b.natT = natT;
    b.nshT = nshT;
    b.naoT = naoT;
    b.nnT = nnT;
    b.npairT = npairT;
    b.nvecT = nvecT;
    b.nsp = nsp;
    b.hist_cap = hist_cap;
    b.m_nat = upI(m_nat);
    b.m_nsh = upI(m_nsh);
    b.m_nao = upI(m_nao);
    b.m_at0 = upI(m_at0);
    b.m_sh0 = upI(m_sh0);
    b.m_ao0 = upI(m_ao0);
    b.m_dim = upI(m_dim);
    b.m_mat0 = upL(m_mat0);
    b.m_gam0 = upL(m_gam0);
    b.m_vec0 = upL(m_vec0);
    b.m_pair0 = upL(m_pair0);
    d_pair0 = const_cast<long long*>(b.m_pair0);
    b.m_hist0 = upL(m_hist0);
    d_pd0 = upL(m_pd0);
    d_tile0 = upL(m_tile0);
    d_sq0 = upL(m_sq0);
    b.m_nalpha = upD(m_na);
    b.m_nbeta = upD(m_nb);
    b.m_charge = upD(m_ch);
    b.a_Z = upI(a_Z);
    b.a_mol = upI(a_mol);
    b.a_sh0 = upI(a_sh0);
    b.a_nsh = upI(a_nsh);
    b.a_ao0 = upI(a_ao0);
    b.a_sp = upI(a_sp);
    b.a_rcov = upD(a_rcov);
    b.a_rad = upD(a_rad);
    b.a_amin = upD(a_amin);
    b.a_rcov_eeq = upD(a_rcov_eeq);
    b.a_en = upD(a_en);
    b.a_aes_rad = upD(a_aes_rad);
    b.a_aes_vcn = upD(a_aes_vcn);
    b.a_dk = upD(a_dk);
    b.a_qk = upD(a_qk);
    b.a_rep_alpha = upD(a_ra);
    b.a_rep_zeff = upD(a_rz);
    b.a_eeq_chi = upD(a_chi);
    b.a_eeq_eta = upD(a_eta);
    b.a_eeq_kcn = upD(a_kcn);
    b.a_eeq_rad = upD(a_erad);
    b.s_l = upI(s_l);
    b.s_np = upI(s_np);
    b.s_at = upI(s_at);
    b.s_ao0 = upI(s_ao0);
    b.s_ish = upI(s_ish);
    b.s_mol = upI(s_mol);
    b.s_Z = upI(s_Z);
    b.s_alpha = upD(s_alpha);
    b.s_coeff = upD(s_coeff);
    b.s_amin = upD(s_amin);
    b.s_se0 = upD(s_se0);
    b.s_kcn = upD(s_kcn);
    b.s_shpoly = upD(s_shpoly);
    b.s_refocc = upD(s_refocc);
    b.s_hard = upD(s_hard);
    b.s_gam3 = upD(s_gam3);
    b.s_slater = upD(s_slater);
    b.o_sh = upI(o_sh);
    b.o_at = upI(o_at);
    b.sp_nref = upI(sp_nref);
    b.sp_ngw = upI(sp_ngw);
    b.sp_refcn = upD(sp_refcn);
    b.sp_refq = upD(sp_refq);
    b.sp_zeff = upD(sp_zeff);
    b.sp_gi = upD(sp_gi);
    b.sp_rcov = upD(sp_rcov);
    b.sp_en = upD(sp_en);
    b.sp_c6ref = upD(c6ref);
    b.sp_rr = upD(sp_rr);
    b.sp_r0 = upD(sp_r0);
    b.intcut = cv.intcut(o.acc);
    // aufbau occupations up to the conventions' temperature (crates/axtb/src/xtb.rs:462)
    b.kt = o.etemp <= cv.aufbau_max_etemp ? 0.0 : o.etemp * cv.kb;
    b.cn_cut = cv.cn_cut;
    b.rep_cut = cv.rep_cut;
    b.d4_cn_cut = cv.d4_cn_cut;
    b.d2_cut = cv.d2_cut;
    b.d2_w = cv.d2_w;
    b.d3_cut = cv.d3_cut;
    b.d3_w = cv.d3_w;
    b.eeq_cn_cut = cv.eeq_cn_cut;
    b.eeq_cap = cv.eeq_cap;
    b.output_aes = cv.output_aes ? 1 : 0;
    {
        vector<double> pc(nmol);
        for (int m = 0; m < nmol; m++) {
            double amin = INFINITY;
            for (int i = 0; i < mols[m].nat; i++) amin = std::min(amin, a_amin[m_at0[m] + i]);
            pc[m] = cv.pair_cut2(o.acc, amin);
        }
        b.m_paircut2 = upD(pc);
    }
    // implicit solvation (crates/solvation/src/lib.rs:394-497 paramToModel and initBorn): axtb's and
    // tblite's conventions use the corrected variant (CODATA 2022 radii and constants), the xtb
    // 6.8.0 conventions xtb's (mctc-lib's bohr factor, xtb's constants in the shift)
    b.solv = o.solv >= 0 ? 1 : 0;
    if (b.solv) {
        using namespace solvtab;
        const SolventParam* p = solvent_param(o.solvent, o.solv == 0);
        bool xtbv = o.conventions == 1;
        double aatoau = xtbv ? 1.0 / 5.29177210904492434e-1 : AATOAU;
        const double temp = DEFAULT_TEMPERATURE;
        auto shift = [&](double kb, double vm) {
            if (o.solv_state == 0) return 0.0;
            double s = std::log(vm * temp / AMBIENT_TEMPERATURE);
            if (o.solv_state == 2) s += std::log(p->rhos / REF_DENSITY * REF_MOLECULAR_MASS / p->smass);
            return temp * kb * s;
        };
        const double hartree_kcal = 4.3597447222060e-18 * 6.02214076e23 / 4184.0;
        const double vm_exact = 6.02214076e23 * 1.380649e-23 * 298.15 / 1.0e5 * 1.0e3;
        b.sv_gshift = xtbv ? p->gshift * (1.0 / AUTOKCAL) + shift(KB, IDEAL_GAS_MOL_VOLUME)
                           : p->gshift / hartree_kcal + shift(KB_HARTREE, vm_exact);
        double eps = p->epsv, offset = p->soset * 0.1 * aatoau, probe = p->rprobe * aatoau;
        bool any_hb = false;
        for (double t : p->tmp) any_hb = any_hb || std::fabs(t) > 1.0e-3;
        b.sv_alpb = o.solv == 0 ? 1 : 0;
        b.sv_alpbet = b.sv_alpb ? ALPB_ALPHA / eps : 0.0;
        b.sv_keps = (1.0 / eps - 1.0) / (1.0 + b.sv_alpbet);
        b.sv_c1 = p->c1;
        b.sv_lrcut = LRCUT_AA * aatoau;
        double w = SMOOTH_W_AA * aatoau, w3 = w * (w * w);
        b.sv_w = w;
        b.sv_ah0 = 0.5;
        b.sv_ah1 = 3.0 / (4.0 * w);
        b.sv_ah3 = -1.0 / (4.0 * w3);
        vector<double> vdwr(natT), rho(natT), svdw(natT), vdwsa(natT), t1(natT), t2(natT), wrp(natT), gam(natT),
            hbmag(natT), srcut(nmol);
        for (int m = 0; m < nmol; m++) {
            double maxsa = -INFINITY;
            for (int i = 0; i < mols[m].nat; i++) {
                int a = m_at0[m] + i, iz = mols[m].Z[i] - 1;
                if (iz + 1 > NELEM) throw Fail(AXTB_ERR_INPUT, "solvation: unsupported element");
                double rvdw = aatoau * VDW_RAD_D3_AA[iz], rsa = rvdw + probe;
                vdwr[a] = rvdw;
                rho[a] = rvdw * p->sx[iz];
                svdw[a] = rvdw - offset;
                vdwsa[a] = rsa;
                maxsa = std::max(maxsa, rsa);
                t1[a] = (rsa - w) * (rsa - w);
                t2[a] = (rsa + w) * (rsa + w);
                double r = rsa + w;
                double wr = (0.25 / w + 3.0 * b.sv_ah3 * (0.2 * r * r - 0.5 * r * rsa + rsa * rsa / 3.0)) * r * r * r;
                r = rsa - w;
                wr -= (0.25 / w + 3.0 * b.sv_ah3 * (0.2 * r * r - 0.5 * r * rsa + rsa * rsa / 3.0)) * r * r * r;
                wrp[a] = wr;
                gam[a] = p->gamscale[iz] * (4.0 * PI_) * SURFACE_TENSION;
                hbmag[a] = any_hb ? -(p->tmp[iz] * p->tmp[iz]) * (1.0 / AUTOKCAL) : 0.0;
            }
            srcut[m] = 2.0 * (w + maxsa) + SRCUT_AA * aatoau;
        }
        b.sv_vdwr = upD(vdwr);
        b.sv_rho = upD(rho);
        b.sv_svdw = upD(svdw);
        b.sv_vdwsa = upD(vdwsa);
        b.sv_t1 = upD(t1);
        b.sv_t2 = upD(t2);
        b.sv_wrp = upD(wrp);
        b.sv_gam = upD(gam);
        b.sv_hbmag = upD(hbmag);
        b.sv_srcut = upD(srcut);
        CK(cudaMemcpyToSymbolAsync(axg::c_lebedev, LEBEDEV_230, sizeof(LEBEDEV_230), 0, cudaMemcpyHostToDevice, st));
    }
    b.damping = o.damping;
    b.econv = 1e-6 * o.acc;
    b.pconv = 2e-5 * o.acc;
    b.max_iter = o.max_iter;
    b.split = o.precision == 1 ? 1 : 0;
    b.disp = o.dispersion ? 1 : 0;
    b.band_max = band_max;
    b.chase_max = chase_max;
    vector<int> pair_off, pair_list, solo_off, solo_list;
    {
        // the plan: pairs (above CHASE_ROWS AOs) on clusters, then the rest one per CTA, longest
        // first onto the least loaded; cost ~ time steps (3 n), a pair's steps ~1.3x a CTA's
        vector<char> is_big(nmol, 0);
        for (int m : big) is_big[m] = 1;
        vector<std::pair<double, int>> pairs, solos;
        for (int m = 0; m < nmol; m++) {
            int n = m_nao[m];
            if (is_big[m] || n <= axg::BW + 1 || n >= b.band_max || n > b.chase_max) continue;
            if (n > axg::CHASE_ROWS) pairs.push_back({3.9 * n, m});
            else solos.push_back({3.0 * n, m});
        }
        nchase = (int)(pairs.size() + solos.size());
        chase_grid = 2 * std::max(1, nsm / 2);
        int ncl = chase_grid / 2;
        auto desc = [](auto& x, auto& y) { return x.first > y.first; };
        std::sort(pairs.begin(), pairs.end(), desc);
        std::sort(solos.begin(), solos.end(), desc);
        using Q = std::priority_queue<std::pair<double, int>, vector<std::pair<double, int>>, std::greater<>>;
        vector<vector<int>> pl(ncl), sl(chase_grid);
        vector<double> load(ncl, 0.0);
        Q qc;
        for (int c = 0; c < ncl; c++) qc.push({0.0, c});
        for (auto& x : pairs) {
            auto top = qc.top();
            qc.pop();
            pl[top.second].push_back(x.second);
            load[top.second] = top.first + x.first;
            qc.push({load[top.second], top.second});
        }
        Q qs;
        for (int g = 0; g < chase_grid; g++) qs.push({load[g / 2], g});
        for (auto& x : solos) {
            auto top = qs.top();
            qs.pop();
            sl[top.second].push_back(x.second);
            qs.push({top.first + x.first, top.second});
        }
        pair_off.assign(ncl + 1, 0);
        for (int c = 0; c < ncl; c++) {
            pair_off[c + 1] = pair_off[c] + (int)pl[c].size();
            for (int m : pl[c]) pair_list.push_back(m);
        }
        solo_off.assign(chase_grid + 1, 0);
        for (int g = 0; g < chase_grid; g++) {
            solo_off[g + 1] = solo_off[g] + (int)sl[g].size();
            for (int m : sl[g]) solo_list.push_back(m);
        }
        pair_list.push_back(0);  // never empty
        solo_list.push_back(0);
    }
    // state
    axg::State& s = S;
    s.xyz = ar.take<double>(natT * 3);
    s.cn = ar.take<double>(natT);
    s.cn_d4 = ar.take<double>(natT);
    s.cn_eeq = ar.take<double>(natT);
    s.mrad = ar.take<double>(natT);
    s.dmrdcn = ar.take<double>(natT);
    s.se = ar.take<double>(nshT);
    s.dsedcn = ar.take<double>(nshT);
    s.S = ar.take<double>(nnT);
    s.H0 = ar.take<double>(nnT);
    s.D = ar.take<double>(nnT * 3);
    s.Q = ar.take<double>(nnT * 6);
    s.Linv = ar.take<double>(nnT);
    s.F = ar.take<double>(nnT);
    s.Fp = ar.take<double>(nnT);
    s.Z = ar.take<double>(nnT);
    s.C = ar.take<double>(nnT);
    s.P = ar.take<double>(nnT);
    s.W = ar.take<double>(nnT);
    s.scr1 = ar.take<double>(nnT);
    s.scr2 = ar.take<double>(nnT);
    s.scr3 = ar.take<double>(nnT);
    s.piv = ar.take<unsigned char>(nnT);
    s.emo = ar.take<double>(naoT);
    s.focc = ar.take<double>(naoT);
    s.focc_a = ar.take<double>(naoT);
    s.efermi = ar.take<double>((size_t)nmol * 2);
    s.dtri = ar.take<double>(naoT);
    s.etri = ar.take<double>(naoT);
    s.tau = ar.take<double>(naoT);
    s.kocc = ar.take<int>(nmol);
    s.status = ar.take<int>(nmol);
    s.conv = ar.take<int>(nmol);
    s.active = ar.take<int>(nmol);
    s.niter = ar.take<int>(nmol);
    s.iter = ar.take<int>(nmol);
    s.mix_used = ar.take<int>(nmol);
    s.niter_prev = ar.take<int>(nmol);
    s.have_guess = ar.take<int>(nmol);
    s.retry = ar.take<int>(nmol);
    CK(cudaMemsetAsync(s.have_guess, 0, sizeof(int) * nmol, st));
    s.diis = ar.take<double>((size_t)nmol * 8);
    s.start = ar.take<double>((size_t)nshT + (size_t)natT * 10);
    s.qsh_in = ar.take<double>(nshT);
    s.qsh_out = ar.take<double>(nshT);
    s.vsh = ar.take<double>(nshT);
    s.qat_in = ar.take<double>(natT);
    s.qat_out = ar.take<double>(natT);
    s.dp_in = ar.take<double>(natT * 3);
    s.dp_out = ar.take<double>(natT * 3);
    s.qp_in = ar.take<double>(natT * 6);
    s.qp_out = ar.take<double>(natT * 6);
    s.vat = ar.take<double>(natT);
    s.vdp = ar.take<double>(natT * 3);
    s.vqp = ar.take<double>(natT * 6);
    s.gw = ar.take<double>(natT * 7);
    s.dgw = ar.take<double>(natT * 7);
    s.ao_part = ar.take<double>((size_t)naoT * 11);
    s.q_in = ar.take<double>(nvecT);
    s.dq = ar.take<double>(nvecT);
    s.qlast = ar.take<double>(nvecT);
    s.dqlast = ar.take<double>(nvecT);
    s.df = ar.take<double>(nhist);
    s.u = ar.take<double>(nhist);
    s.amat = ar.take<double>((size_t)nmol * hist_cap * hist_cap * 2);
    s.omega = ar.take<double>((size_t)nmol * hist_cap);
    s.energy = ar.take<double>(nmol);
    s.elast = ar.take<double>(nmol);
    s.de = ar.take<double>(nmol);
    s.res = ar.take<double>(nmol);
    s.ts = ar.take<double>(nmol);
    s.e_fixed = ar.take<double>(nmol);
    s.terms = ar.take<double>((size_t)nmol * 8);
    s.grad = ar.take<double>(natT * 3);
    s.dedcn = ar.take<double>(natT);
    s.dedcn_d4 = ar.take<double>(natT);
    s.pair_buf = ar.take<double>((size_t)std::max(npairT, 1LL) * 5);
    s.e_atom = ar.take<double>(natT);
    s.e_terms = ar.take<double>(natT * 5);
    s.mol_cyc = ar.take<double>(nmol);
    if (o.solv >= 0) {
        s.sv_brad = ar.take<double>(natT);
        s.sv_dbrad = ar.take<double>(natT);
        s.sv_sasa = ar.take<double>(natT);
        s.sv_hbw = ar.take<double>(natT);
        s.sv_dhbdw = ar.take<double>(natT);
        s.sv_selfg = ar.take<double>((size_t)natT * 3);
        s.sv_dedbr = ar.take<double>(natT);
        s.sv_adet = ar.take<double>(nmol);
        s.sv_eatom = ar.take<double>(natT);
        s.sv_emol = ar.take<double>(nmol);
        s.sv_nb = ar.take<int>((size_t)natT * axg::SOLV_MAXNB);
        s.sv_nbn = ar.take<int>(natT);
    }
    s.red = ar.take<double>((size_t)axg::team_red_doubles(grid));  // grid-team partials
    s.eeq_A = ar.take<double>((size_t)nsqT * 3);
    s.gam = ar.take<double>((size_t)std::max(ngamT, 1LL));
    // team plan
    P.big = upI(big);
    P.nbig = (int)big.size();
    P.small_off = upI(small_off);
    P.small_list = upI(small_list);
    P.head_off = upI(head_off);
    P.head_list = upI(head_list);
    P.tail_off = upI(tail_off);
    P.tail_list = upI(tail_list);
    CP.pair_off = upI(pair_off);
    CP.pair_list = upI(pair_list);
    CP.solo_off = upI(solo_off);
    CP.solo_list = upI(solo_list);
    P.m_wk0 = upL(m_wk0);
    P.wk = ar.take<double>(nwk);
    P.m_sq0 = d_sq0;
    P.eeq_rhs = ar.take<double>(natT);
    P.eeq_q = ar.take<double>(natT);
    P.eeq_plane = nsqT;
    d_wt = ar.take<double>(std::max(nsqT, 1LL));
    d_tt = ar.take<double>(std::max(nsqT, 1LL));
    d_eatm = ar.take<double>(nmol);
    e_rep.assign(nmol, 0.0);
    e_atm.assign(nmol, 0.0);
    CK(cudaMallocHost(&h_act, sizeof(int) * nmol));
    h_stage_len = std::max<size_t>((size_t)natT * 12 + (size_t)nshT + (size_t)nmol * 16, 1024);
    CK(cudaMallocHost(&h_stage, sizeof(double) * h_stage_len));
    CK(cudaStreamSynchronize(st));
}

// ------------------------------------------------------------------ small kernels of the driver
namespace axg {

// per-molecule sum of an atom array (one CTA per molecule)
__global__ void k_mol_sum(Batch B, const double* src, double* dst) {
    int m = blockIdx.x;
    if (m >= B.nmol) return;
    double s = 0.0;
    for (int a = threadIdx.x; a < B.m_nat[m]; a += blockDim.x) s += src[B.m_at0[m] + a];
    s = cta_sum(s);
    if (threadIdx.x == 0) dst[m] = s;
}

// the first attempt of molecule m starts here: counters, the mixer of the attempt (0 Broyden,
// 1 DIIS) and a copy of the start moments for a later attempt from the same start
__device__ void begin_attempts(const Batch& B, const State& S, int m, int mixer) {
    int a0 = B.m_at0[m], nat = B.m_nat[m], s0 = B.m_sh0[m], nsh = B.m_nsh[m];
    double* st_sh = S.start;
    double* st_at = S.start + B.nshT;
    for (int s = s0 + threadIdx.x; s < s0 + nsh; s += blockDim.x) st_sh[s] = S.qsh_in[s];
    for (int a = a0 + threadIdx.x; a < a0 + nat; a += blockDim.x) {
        double* t = st_at + 10LL * a;
        t[0] = S.qat_in[a];
        for (int k = 0; k < 3; k++) t[1 + k] = S.dp_in[3 * a + k];
        for (int k = 0; k < 6; k++) t[4 + k] = S.qp_in[6 * a + k];
    }
    __syncthreads();
    pack_moment(B, m, S.qsh_in, S.dp_in, S.qp_in, S.q_in + B.m_vec0[m], threadIdx.x, blockDim.x);
    if (threadIdx.x == 0) {
        S.elast[m] = 0.0;
        S.iter[m] = 0;
        S.niter[m] = 0;
        S.niter_prev[m] = 0;
        S.conv[m] = 0;
        S.mix_used[m] = mixer == 2 ? 1 : 0;
        diis_reset(B, S, m);
        S.active[m] = S.status[m] == 0 ? 1 : 0;
    }
}

// start moments: EEQ charges split over the shells by reference occupation
// (crates/axtb/src/xtb.rs:522-549), zero multipoles, packed SCC vector
__global__ void k_start(Batch B, State S, const double* qeeq, int use_eeq, int mixer, const int* only) {
    int m = blockIdx.x;
    if (m >= B.nmol || (only && !only[m])) return;
    if (only && threadIdx.x == 0) S.status[m] = 0;  // a fresh retry forgets the failed attempt
    int a0 = B.m_at0[m], nat = B.m_nat[m];
    for (int a = a0 + threadIdx.x; a < a0 + nat; a += blockDim.x) {
        double tot = 0.0;
        for (int s = B.a_sh0[a]; s < B.a_sh0[a] + B.a_nsh[a]; s++) tot += B.s_refocc[s];
        double qa = 0.0;
        for (int s = B.a_sh0[a]; s < B.a_sh0[a] + B.a_nsh[a]; s++) {
            double q = (use_eeq && tot > 0.0) ? qeeq[a] * B.s_refocc[s] / tot : 0.0;
            S.qsh_in[s] = q;
            qa += q;
        }
        S.qat_in[a] = qa;
        for (int k = 0; k < 3; k++) S.dp_in[3 * a + k] = 0.0;
        for (int k = 0; k < 6; k++) S.qp_in[6 * a + k] = 0.0;
    }
    __syncthreads();
    begin_attempts(B, S, m, mixer);
}

// start of a warm SCF: the previous converged output moments of every molecule (of those with
// only[m] set)
__global__ void k_start_warm(Batch B, State S, int mixer, const int* only) {
    int m = blockIdx.x;
    if (m >= B.nmol || (only && !only[m])) return;
    int a0 = B.m_at0[m], nat = B.m_nat[m], s0 = B.m_sh0[m], nsh = B.m_nsh[m];
    for (int s = s0 + threadIdx.x; s < s0 + nsh; s += blockDim.x) S.qsh_in[s] = S.qsh_out[s];
    for (int a = a0 + threadIdx.x; a < a0 + nat; a += blockDim.x) {
        S.qat_in[a] = S.qat_out[a];
        for (int k = 0; k < 3; k++) S.dp_in[3 * a + k] = S.dp_out[3 * a + k];
        for (int k = 0; k < 6; k++) S.qp_in[6 * a + k] = S.qp_out[6 * a + k];
    }
    __syncthreads();
    begin_attempts(B, S, m, mixer);
}

// the DIIS attempt of the auto plan (crates/axtb/src/xtb.rs:590-645): a molecule whose Broyden
// attempt ended unconverged, with a failed mixer or a lost Fermi level starts again from its
// start moments with DIIS; one that ended with an error axtb raises at once does not. Within an
// iteration axtb checks the Fock matrix (non-finite: error), then the Fermi level (lost: next
// attempt, crates/axtb/src/xtb.rs:1013-1025), then the energy (non-finite: error); the eigen
// phase here goes on after a lost Fermi level, so bits it sets after one do not count. The
// iterations of the Broyden attempt are kept for the failure report.
__global__ void k_restart_diis(Batch B, State S) {
    int m = blockIdx.x;
    if (m >= B.nmol) return;
    __shared__ int s_go;
    if (threadIdx.x == 0) {
        int st = S.status[m];
        bool hard = (st & (ST_NOT_PD | ST_FOCK | ST_TIMEOUT)) != 0 ||
                    (!(st & ST_FERMI) && (st & (ST_NONFINITE | ST_INVIT)) != 0);
        s_go = !S.conv[m] && !hard && S.mix_used[m] == 0;  // a Broyden attempt that just ended
    }
    __syncthreads();
    if (!s_go) return;
    int a0 = B.m_at0[m], nat = B.m_nat[m], s0 = B.m_sh0[m], nsh = B.m_nsh[m];
    const double* st_sh = S.start;
    const double* st_at = S.start + B.nshT;
    for (int s = s0 + threadIdx.x; s < s0 + nsh; s += blockDim.x) S.qsh_in[s] = st_sh[s];
    for (int a = a0 + threadIdx.x; a < a0 + nat; a += blockDim.x) {
        const double* t = st_at + 10LL * a;
        S.qat_in[a] = t[0];
        for (int k = 0; k < 3; k++) S.dp_in[3 * a + k] = t[1 + k];
        for (int k = 0; k < 6; k++) S.qp_in[6 * a + k] = t[4 + k];
    }
    __syncthreads();
    pack_moment(B, m, S.qsh_in, S.dp_in, S.qp_in, S.q_in + B.m_vec0[m], threadIdx.x, blockDim.x);
    if (threadIdx.x == 0) {
        S.niter_prev[m] = S.niter[m];
        S.elast[m] = 0.0;
        S.iter[m] = 0;
        S.niter[m] = 0;
        S.conv[m] = 0;
        S.status[m] = 0;
        S.mix_used[m] = 2;
        diis_reset(B, S, m);
        S.active[m] = 1;
    }
}

// molecules that started from their previous moments and ended unconverged run once more from
// the fresh guess (crates/axtb/src/calculator.rs:194-206, RetryLadder::warm_then_fresh, which
// climbs on ScfNotConverged only: crates/base/src/method/retry.rs:119-158)
__global__ void k_fresh_mask(Batch B, State S) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= B.nmol) return;
    S.retry[m] = S.have_guess[m] && !S.conv[m] && (S.status[m] & ~ST_HISTORY) == 0;
}

}  // namespace axg

namespace {

inline unsigned blocks_for(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// positions of every molecule into HBM: from a device pointer directly, from host memory
// through the pinned staging buffer
void AxtbBatch::upload_positions(const double* x, bool device_ptr) {
    size_t bytes = sizeof(double) * 3 * natT;
    if (device_ptr) {
        CK(cudaMemcpyAsync(S.xyz, x, bytes, cudaMemcpyDeviceToDevice, st));
        return;
    }
    std::memcpy(h_stage, x, bytes);
    CK(cudaMemcpyAsync(S.xyz, h_stage, bytes, cudaMemcpyHostToDevice, st));
    h2d_bytes += (long long)bytes;
}

// Optional per-launch timing: CUDA events recorded on the batch stream around each kernel,
// resolved after the run; with the algorithmic work of each launch (FLOPs of the dense algebra,
// bytes of the matrix passes) for the roofline report.
void AxtbBatch::begin_launch(const char* name, double flops, double bytes) {
    launches++;
    if (!profiling) return;
    Rec r;
    r.name = name;
    r.flops = flops;
    r.bytes = bytes;
    CK(cudaEventCreate(&r.e0));
    CK(cudaEventCreate(&r.e1));
    CK(cudaEventRecord(r.e0, st));
    recs.push_back(r);
}

void AxtbBatch::end_launch() {
    if (!profiling) return;
    CK(cudaEventRecord(recs.back().e1, st));
}

void AxtbBatch::resolve_profile() {
    if (!profiling) return;
    CK(cudaStreamSynchronize(st));
    unsigned long long cyc[axg::TEAM_CYCLE_SLOTS];
    CK(cudaMemcpyFromSymbol(cyc, axg::g_team_cycles, sizeof cyc));
    for (int k = 0; k < axg::TEAM_CYCLE_SLOTS; k++) team_cycles[k] += (double)cyc[k];
    eigen_ms.clear();
    for (auto& r : recs) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, r.e0, r.e1));
        if (std::strcmp(r.name, "team_eigen") == 0) eigen_ms.push_back(ms);
        auto& a = prof[r.name];
        a.launches += 1;
        a.ms += ms;
        a.flops += r.flops;
        a.bytes += r.bytes;
        cudaEventDestroy(r.e0);
        cudaEventDestroy(r.e1);
    }
    recs.clear();
}

void AxtbBatch::run(bool want_grad, bool warm, bool want_levels) {
    using namespace axg;
    launches = 0;
    h_warm.assign(nmol, warm ? 1 : 0);
    CK(cudaEventRecord(phase_ev[0], st));
    P.cycles = profiling ? 1 : 0;
    if (profiling) {
        unsigned long long z[TEAM_CYCLE_SLOTS] = {0};
        CK(cudaMemcpyToSymbolAsync(g_team_cycles, z, sizeof z, 0, cudaMemcpyHostToDevice, st));
    }
    const int T = 256;
    long long nn = nnT;
#define LAUNCH(name, flops, bytes, ...)  \
    do {                                 \
        begin_launch(name, flops, bytes); \
        __VA_ARGS__;                     \
        end_launch();                    \
    } while (0)
    // algorithmic work of the matrix passes over the molecules in `act` (1 = included)
    auto mat_bytes = [&](const vector<int>& act, double per_n2) {
        double s = 0.0;
        for (int m = 0; m < nmol; m++)
            if (act[m]) s += per_n2 * 8.0 * (double)mols[m].nao * mols[m].nao;
        return s;
    };
    auto eig_flops = [&](const vector<int>& act) {
        double s = 0.0;
        for (int m = 0; m < nmol; m++)
            if (act[m]) {
                double n = mols[m].nao, k = std::ceil(mols[m].nalpha);
                // algorithmic count: n^3 (reduction to standard form, sygst), 4/3 n^3
                // (tridiagonalisation), 2 n^2 k (Householder back-transform), n^2 k (L^-T) and
                // n^2 k (P); the work the kernel does beyond this is overhead, not counted
                s += n * n * n + 4.0 / 3.0 * n * n * n + 4.0 * n * n * k;
            }
        return s;
    };
    auto w_flops = [&](const vector<int>& act) {
        double s = 0.0;
        for (int m = 0; m < nmol; m++)
            if (act[m]) s += 2.0 * mols[m].nao * mols[m].nao * std::ceil(mols[m].nalpha);
        return s;
    };
    vector<int> all(nmol, 1), act(nmol, 1);
    // reset per-run state
    CK(cudaMemsetAsync(S.status, 0, sizeof(int) * nmol, st));
    CK(cudaMemsetAsync(S.S, 0, sizeof(double) * nn * 11, st));  // S, H0, D(3), Q(6) contiguous
    CK(cudaMemsetAsync(S.grad, 0, sizeof(double) * natT * 3, st));
    CK(cudaMemsetAsync(S.dedcn, 0, sizeof(double) * natT, st));
    CK(cudaMemsetAsync(S.dedcn_d4, 0, sizeof(double) * natT, st));
    CK(cudaMemsetAsync(S.e_atom, 0, sizeof(double) * natT, st));
    CK(cudaMemsetAsync(S.terms, 0, sizeof(double) * nmol * 8, st));
    CK(cudaMemsetAsync(S.ts, 0, sizeof(double) * nmol, st));
    // geometry
    LAUNCH("cn", 0, 0, k_cn<<<blocks_for((long long)natT * 32, T), T, 0, st>>>(B, S));
    if (ngamT > 0) LAUNCH("gamma", 0, 0, k_gamma<<<blocks_for(ngamT, T), T, 0, st>>>(B, S, ngamT));
    LAUNCH("selfenergy", 0, 0, k_selfenergy<<<blocks_for(std::max(natT, nshT), T), T, 0, st>>>(B, S));
    LAUNCH("repulsion", 0, 0, k_repulsion<<<blocks_for((long long)natT * 32, T), T, 0, st>>>(B, S));
    LAUNCH("mol_sum", 0, 0, k_mol_sum<<<nmol, T, 0, st>>>(B, S.e_atom, S.e_fixed));
    CK(cudaMemsetAsync(S.e_atom, 0, sizeof(double) * natT, st));
    // D4 three-body at q = 0 with dgw/dCN weights (none without the D4 term)
    if (B.disp) {
        CK(cudaMemsetAsync(P.eeq_q, 0, sizeof(double) * natT, st));
        LAUNCH("d4_weights", 0, 0, k_d4_weights<<<blocks_for(natT, T), T, 0, st>>>(B, S, P.eeq_q, 1));
        LAUNCH("atm_tables", 0, 0, k_atm_tables<<<blocks_for(nsqT, T), T, 0, st>>>(B, S, d_wt, d_tt, d_sq0, nsqT));
        if (npairT > 0)
            LAUNCH("atm", 0, 0,
                   k_atm_pairs<<<blocks_for(npairT * 32, T), T, 0, st>>>(B, S, d_wt, d_tt, d_sq0, d_pair0, npairT,
                                                                        S.pair_buf));
        LAUNCH("atm_gather", 0, 0, k_atm_gather<<<blocks_for((long long)natT * 32, T), T, 0, st>>>(B, S, d_pair0, S.pair_buf));
        LAUNCH("mol_sum", 0, 0, k_mol_sum<<<nmol, T, 0, st>>>(B, S.e_atom, d_eatm));
    } else {
        CK(cudaMemsetAsync(d_eatm, 0, sizeof(double) * nmol, st));
    }
    // integrals
    LAUNCH("integrals", 0, mat_bytes(all, 11.0), k_integrals<<<blocks_for(npdT, 128), 128, 0, st>>>(B, S, d_pd0, npdT));
    if (B.solv) {  // solvation: Born radii, SASA neighbours and surfaces, ALPB shape descriptor
        unsigned wb = blocks_for((long long)natT * 32, T);
        LAUNCH("solv_born", 0, 0, k_solv_born<<<wb, T, 0, st>>>(B, S));
        LAUNCH("solv_neighbours", 0, 0, k_solv_neighbours<<<wb, T, 0, st>>>(B, S));
        LAUNCH("solv_sasa", 0, 0, k_solv_sasa<<<wb, T, 0, st>>>(B, S));
        LAUNCH("solv_adet", 0, 0, k_solv_adet<<<nmol, 32, 0, st>>>(B, S));
    }
    // overlap factorisation and EEQ start
    void* args[] = {&B, &S, &P, nullptr};
    int ph = PH_OVERLAP;
    args[3] = &ph;
    // a team phase: the whole-grid molecules in their own launch (k_team_grid), then the rest
    TeamPlan Psmall = P;
    Psmall.nbig = 0;
    void* args_small[] = {&B, &S, &Psmall, &ph};
    auto team_launch = [&](int phase) {
        ph = phase;
        Psmall = P;
        Psmall.nbig = 0;
        if (P.nbig > 0 && phase != PH_EIGEN_TAIL) {  // no whole-grid molecule has a part after k_chase
            CK(cudaLaunchCooperativeKernel((void*)k_team_grid, grid, TEAM_THREADS, args, SMEM_WORK_BYTES, st));
            launches++;
        }
        CK(cudaLaunchCooperativeKernel((void*)k_team, grid, TEAM_THREADS, args_small, SMEM_WORK_BYTES, st));
    };
    double chol_flops = 0.0;
    for (int m = 0; m < nmol; m++) chol_flops += (1.0 / 3.0 + 2.0 / 3.0) * std::pow((double)mols[m].nao, 3.0);
    LAUNCH("team_overlap", chol_flops, 0,
           team_launch(PH_OVERLAP));
    bool eeq = opt.guess == 0 && eeq_guess && !warm;
    if (warm) {
        LAUNCH("start", 0, 0, k_start_warm<<<nmol, T, 0, st>>>(B, S, mixer_kind, nullptr));
    } else if (eeq) {
        LAUNCH("eeq_matrix", 0, 0, k_eeq_matrix<<<blocks_for(nsqT, T), T, 0, st>>>(B, S, d_sq0, P.eeq_rhs, nsqT));
        double f = 0.0;
        for (int m = 0; m < nmol; m++) f += 3.0 * std::pow((double)mols[m].nat, 3.0);
        LAUNCH("team_eeq", f, 0, team_launch(PH_EEQ));
    }
    if (!warm) LAUNCH("start", 0, 0, k_start<<<nmol, T, 0, st>>>(B, S, P.eeq_q, eeq ? 1 : 0, mixer_kind, nullptr));
    // restarts: a molecule with converged moments from the previous run starts from them
    if (restart && !warm)
        LAUNCH("start_warm", 0, 0, k_start_warm<<<nmol, T, 0, st>>>(B, S, mixer_kind, S.have_guess));
    // SCF: the attempts of the mixer plan (crates/axtb/src/scf/mixing.rs:163-199): Broyden, then
    // for the molecules it left unconverged DIIS from the same start (auto); or one mixer alone
    auto scf_attempt = [&](bool diis) {
        for (int it = 1; it <= opt.max_iter; it++) {
            LAUNCH("d4_weights", 0, 0, k_d4_weights<<<blocks_for(natT, T), T, 0, st>>>(B, S, S.qat_in, 0));
            LAUNCH("potentials", 0, 0, k_potentials<<<blocks_for((long long)natT * 32, T), T, 0, st>>>(B, S));
            if (B.solv)
                LAUNCH("solv_potential", 0, 0, k_solv_potential<<<blocks_for((long long)natT * 32, T), T, 0, st>>>(B, S));
            LAUNCH("fock", 0, mat_bytes(act, 12.0), k_fock<<<(unsigned)ntiles, T, 0, st>>>(B, S, d_tile0, ntiles));
            // the eigen phase: one launch, or three when k_chase takes stage 2 of some molecules
            LAUNCH("team_eigen", eig_flops(act), 0, {
                team_launch(PH_EIGEN);
                if (nchase > 0) {
                    CP.cycles = P.cycles;
                    k_chase<<<chase_grid, CHASE_THREADS, CHASE_DYN_BYTES, st>>>(B, S, CP);
                    CK(cudaGetLastError());
                    team_launch(PH_EIGEN_TAIL);
                    launches += 2;
                }
            });
            LAUNCH("mulliken", 0, mat_bytes(act, 12.0),
                   k_mulliken<<<blocks_for((long long)naoT * 32, T), T, 0, st>>>(B, S));
            LAUNCH("moments", 0, 0, k_moments<<<blocks_for(natT, T), T, 0, st>>>(B, S));
            LAUNCH("d4_weights", 0, 0, k_d4_weights<<<blocks_for(natT, T), T, 0, st>>>(B, S, S.qat_out, 2));
            LAUNCH("energy", 0, 0, k_energy<<<blocks_for((long long)natT * 32, T), T, 0, st>>>(B, S));
            if (B.solv)
                LAUNCH("solv_energy", 0, 0, k_solv_energy<<<blocks_for((long long)natT * 32, T), T, 0, st>>>(B, S));
            if (diis) LAUNCH("diis", 0, 0, k_diis<<<nmol, T, 0, st>>>(B, S));
            else LAUNCH("broyden", 0, 0, k_broyden<<<nmol, T, 0, st>>>(B, S, hist_cap));
            CK(cudaMemcpyAsync(h_act, S.active, sizeof(int) * nmol, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            std::copy(h_act, h_act + nmol, act.begin());
            if (std::none_of(act.begin(), act.end(), [](int v) { return v != 0; })) break;
        }
    };
    auto scf_plan = [&]() {
        scf_attempt(mixer_kind == 2);
        if (mixer_kind == 0) {
            LAUNCH("restart_diis", 0, 0, k_restart_diis<<<nmol, T, 0, st>>>(B, S));
            CK(cudaMemcpyAsync(h_act, S.active, sizeof(int) * nmol, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            std::copy(h_act, h_act + nmol, act.begin());
            if (std::any_of(act.begin(), act.end(), [](int v) { return v != 0; })) scf_attempt(true);
        }
    };
    CK(cudaEventRecord(phase_ev[1], st));
    if (restart && !warm) {
        CK(cudaMemcpyAsync(h_act, S.have_guess, sizeof(int) * nmol, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        std::copy(h_act, h_act + nmol, h_warm.begin());
    }
    scf_plan();
    if (restart && !warm) {
        // warm starts that did not converge: the whole plan once more from the fresh guess
        // (not for the displaced points of a numerical Hessian, which report the failure)
        bool again = false;
        if (retry_fresh) {
            LAUNCH("fresh_mask", 0, 0, k_fresh_mask<<<blocks_for(nmol, T), T, 0, st>>>(B, S));
            CK(cudaMemcpyAsync(h_act, S.retry, sizeof(int) * nmol, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            again = std::any_of(h_act, h_act + nmol, [](int v) { return v != 0; });
        }
        if (again) {
            for (int m = 0; m < nmol; m++)
                if (h_act[m]) h_warm[m] = 0;
            LAUNCH("start", 0, 0, k_start<<<nmol, T, 0, st>>>(B, S, P.eeq_q, eeq ? 1 : 0, mixer_kind, S.retry));
            CK(cudaMemcpyAsync(h_act, S.active, sizeof(int) * nmol, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            std::copy(h_act, h_act + nmol, act.begin());
            scf_plan();
        }
        // the converged moments are the next run's starts
        CK(cudaMemcpyAsync(S.have_guess, S.conv, sizeof(int) * nmol, cudaMemcpyDeviceToDevice, st));
    }
    if (want_levels) {
        LAUNCH("team_levels", 0, 0, team_launch(PH_LEVELS));
    }
    CK(cudaEventRecord(phase_ev[2], st));
    if (want_grad) {
        LAUNCH("team_wdens", w_flops(all), 0, team_launch(PH_WDENS));
        if (B.output_aes)
            LAUNCH("gradient_potentials", 0, 0,
                   k_gradient_potentials_aes<<<blocks_for((long long)natT * 32, T), T, 0, st>>>(B, S));
        if (npairT > 0)
            LAUNCH("h0_gradient", 0, mat_bytes(all, 2.0),
                   k_h0_gradient<<<blocks_for(npairT, 128), 128, 0, st>>>(B, S, d_pair0, npairT, S.pair_buf));
        LAUNCH("h0_gather", 0, 0, k_h0_gather<<<blocks_for((long long)natT * 32, T), T, 0, st>>>(B, S, d_pair0, S.pair_buf));
        LAUNCH("d4_weights", 0, 0, k_d4_weights<<<blocks_for(natT, T), T, 0, st>>>(B, S, S.qat_out, 1));
        LAUNCH("grad_pairs", 0, 0, k_grad_pairs<<<blocks_for((long long)natT * 32, T), T, 0, st>>>(B, S));
        if (B.solv) {
            unsigned wb = blocks_for((long long)natT * 32, T);
            LAUNCH("solv_grad_kernel", 0, 0, k_solv_grad_kernel<<<wb, T, 0, st>>>(B, S));
            LAUNCH("solv_grad_psi", 0, 0, k_solv_grad_psi<<<wb, T, 0, st>>>(B, S));
            LAUNCH("solv_grad_surface", 0, 0, k_solv_grad_surface<<<wb, T, 0, st>>>(B, S));
            LAUNCH("solv_grad_adet", 0, 0, k_solv_grad_adet<<<nmol, T, 0, st>>>(B, S));
        }
        LAUNCH("cn_chain", 0, 0, k_cn_chain<<<blocks_for((long long)natT * 32, T), T, 0, st>>>(B, S));
    }
#undef LAUNCH
    CK(cudaEventRecord(phase_ev[3], st));
    CK(cudaGetLastError());
    resolve_profile();
}

// ------------------------------------------------------------------ allocation-free density
// Eigenvalues, Fermi occupations and density of one molecule from its Fock and overlap
// matrices (the team kernel's overlap and eigen phases on one CTA) with every scratch buffer in
// one file-scope device array instead of memory from cudaMalloc: for callers that cannot
// allocate device memory themselves (code running inside another framework's stream-ordered
// memory pool or under a fixed device-memory budget, where a cudaMalloc would fail or would
// synchronise the device and stall unrelated work). The array exists once per device for as
// long as the library is loaded; it bounds the molecule to STATIC_MAX_NAO basis functions.
namespace {
constexpr int STATIC_MAX_NAO = 256;
constexpr long long STATIC_PLANE = (long long)STATIC_MAX_NAO * STATIC_MAX_NAO;  // doubles per matrix
constexpr long long STATIC_WK = axg::team_workspace(STATIC_MAX_NAO);             // team workspace
static_assert(STATIC_WK >= axg::band_workspace(STATIC_MAX_NAO) && STATIC_WK >= axg::onestage_workspace(STATIC_MAX_NAO),
              "the static workspace holds the eigen phase's layout at the largest molecule");
constexpr long long STATIC_VEC = 8LL * STATIC_MAX_NAO;                           // d, e, tau + spare
constexpr long long STATIC_PIV = STATIC_PLANE / 8;                               // pivot bytes, as doubles
constexpr long long STATIC_PAR = 64;                                             // small parameters
constexpr long long STATIC_DOUBLES = 8 * STATIC_PLANE + STATIC_WK + STATIC_VEC + STATIC_PIV + STATIC_PAR;
static __device__ __align__(256) double g_density_scratch[STATIC_DOUBLES];  // 4.89 MiB

std::mutex g_static_mu;
double* g_static_addr[256] = {nullptr};
}  // namespace

namespace axg {
// one CTA: parameters into the static area, then the factorisation and the eigen phase
__global__ void __launch_bounds__(TEAM_THREADS)
    k_density_static(Batch B, State S, TeamPlan P, int nao, double nalpha, double nbeta, int* d_status) {
    if (threadIdx.x == 0) {
        *const_cast<int*>(B.m_nao) = nao;
        *const_cast<int*>(B.m_ao0) = 0;
        *const_cast<long long*>(B.m_mat0) = 0;
        *const_cast<long long*>(P.m_wk0) = 0;
        *const_cast<double*>(B.m_nalpha) = nalpha;
        *const_cast<double*>(B.m_nbeta) = nbeta;
        S.status[0] = 0;  // the array keeps the previous call's words
        S.kocc[0] = 0;
    }
    __syncthreads();
    Team one{0, 1, false};
    mol_overlap(one, B, S, P, 0);
    mol_eigen(one, B, S, P, 0, false);
    mol_levels(one, B, S, P, 0);  // every orbital energy, not only the ones the filling needs
    if (threadIdx.x == 0 && d_status) *d_status = S.status[0];
}
}  // namespace axg

extern "C" int axtb_gpu_density_static(const double* d_fock, const double* d_overlap, int32_t nao, double nalpha,
                                       double nbeta, double kt, double* d_emo, double* d_focc, double* d_density,
                                       int32_t* d_status, void* stream) {
    if (!d_fock || !d_overlap || !d_emo || !d_focc || !d_density) {
        g_last_error = "axtb_gpu_density_static: null pointer argument";
        return AXTB_ERR_INPUT;
    }
    if (nao <= 0 || nao > STATIC_MAX_NAO) {
        g_last_error = "axtb_gpu_density_static: nao must be in 1.." + std::to_string(STATIC_MAX_NAO) + ", got " +
                       std::to_string(nao);
        return AXTB_ERR_INPUT;
    }
    if (!(nalpha >= 0.0 && nbeta >= 0.0 && nalpha <= nao && nbeta <= nao) || !(kt >= 0.0)) {
        g_last_error = "axtb_gpu_density_static: electron counts must be in [0, nao] and kT >= 0";
        return AXTB_ERR_INPUT;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) {
        g_last_error = "axtb_gpu_density_static: no current CUDA device";
        return AXTB_ERR_DEVICE;
    }
    double* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_static_mu);
        if (!g_static_addr[dev]) {
            // host code only holds a stand-in for the array: its device address comes from the
            // runtime, once per device, with that device current
            cudaError_t e = cudaGetSymbolAddress((void**)&g_static_addr[dev], g_density_scratch);
            if (e == cudaSuccess)  // the kernel's dynamic shared work area (no device allocation)
                e = cudaFuncSetAttribute((const void*)axg::k_density_static, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         axg::SMEM_WORK_BYTES);
            if (e != cudaSuccess) {
                g_static_addr[dev] = nullptr;
                g_last_error = std::string("axtb_gpu_density_static: device set-up: ") + cudaGetErrorString(e);
                return AXTB_ERR_DEVICE;
            }
        }
        base = g_static_addr[dev];
    }
    double* p = base;
    auto take = [&](long long n) {
        double* r = p;
        p += n;
        return r;
    };
    axg::Batch B{};
    axg::State S{};
    axg::TeamPlan P{};
    S.scr1 = take(STATIC_PLANE);
    S.Linv = take(STATIC_PLANE);
    S.Fp = take(STATIC_PLANE);
    S.Z = take(STATIC_PLANE);
    S.C = take(STATIC_PLANE);
    S.scr2 = take(STATIC_PLANE);
    S.scr3 = take(STATIC_PLANE);
    S.W = take(STATIC_PLANE);  // the band reduction's second-stage reflectors
    P.wk = take(STATIC_WK);
    double* vec = take(STATIC_VEC);
    S.dtri = vec;
    S.etri = vec + STATIC_MAX_NAO;
    S.tau = vec + 2 * STATIC_MAX_NAO;
    S.piv = reinterpret_cast<unsigned char*>(take(STATIC_PIV));
    double* par = take(STATIC_PAR);
    B.m_nao = reinterpret_cast<const int*>(par + 0);
    B.m_ao0 = reinterpret_cast<const int*>(par + 1);
    B.m_mat0 = reinterpret_cast<const long long*>(par + 2);
    P.m_wk0 = reinterpret_cast<const long long*>(par + 3);
    B.m_nalpha = par + 4;
    B.m_nbeta = par + 5;
    S.ts = par + 6;
    S.kocc = reinterpret_cast<int*>(par + 7);
    S.status = reinterpret_cast<int*>(par + 8);
    S.red = par + 16;
    S.S = const_cast<double*>(d_overlap);
    S.F = const_cast<double*>(d_fock);
    S.emo = d_emo;
    S.focc = d_focc;
    S.P = d_density;
    B.nmol = 1;
    B.kt = kt;
    B.band_max = STATIC_BAND_MAX_NAO;
    B.chase_max = 0;  // stage 2 in this kernel
    axg::k_density_static<<<1, axg::TEAM_THREADS, axg::SMEM_WORK_BYTES, (cudaStream_t)stream>>>(B, S, P, nao, nalpha, nbeta,
                                                                                              d_status);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        g_last_error = std::string("axtb_gpu_density_static: launch: ") + cudaGetErrorString(e);
        return AXTB_ERR_DEVICE;
    }
    return AXTB_OK;
}

#include "../../include/axtb_gpu_debug.h"
#include "capi.cuh"
