// Front and back end of the map engine: GPF keyword handling, receptor PDBQT
// reader, energy tables, bond vectors / disorder flags, and the .fld/.xyz/.map
// writers.  Behaviour mirrors AutoGrid 4.2.8's main() (main.cpp:214-2776 and
// :3481-3582); each step cites the lines it restates.  State lives in a Job
// object instead of function-local statics, and fatal conditions raise
// agb::Fatal instead of calling exit().
#include <algorithm>
#include <array>
#include <cctype>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <memory>
#include <string>
#include <thread>
#include <vector>
#include <strings.h>

#include "frontend.hpp"

namespace agb {

static thread_local std::string g_last_error;
void set_last_error(const std::string &m) { g_last_error = m; }
const char *last_error() { return g_last_error.c_str(); }

namespace {

constexpr double kApproxZero = 1.0e-6;   // autocomm.h:72
constexpr double kEintClamp = 100000.;   // autocomm.h:89
constexpr double kFactor = 332.0;        // main.cpp:561
constexpr double kBig = 1.0e12;          // sentinel for extents
constexpr double kPrecision = 0.0001;    // autogrid.h:68
constexpr int kMaxNBonds = 4;            // autogrid.h:59
const char *kProgram = "autogrid4_b200";

enum Kw {
    K_UNKNOWN = -1, K_NULL, K_COMMENT, K_RECEPTOR, K_GRIDFLD, K_NPTS, K_SPACING, K_GRIDCENTER,
    K_LIGAND_TYPES, K_MAP, K_NBP_COEFFS, K_NBP_R_EPS, K_ELECMAP, K_DIEL, K_FMAP, K_DISORDER,
    K_SMOOTH, K_SOL_PAR, K_CONSTANT, K_COVALENTMAP, K_RECEPTOR_TYPES, K_PARAM_FILE, K_DSOLVMAP,
    K_QASP, K_USE_VINA, K_OUTLEV, K_MAP_RECEPTOR_INTERIOR, K_CMAP, K_CONSTRICTION_CUTOFF,
    K_SEPARATE_DESOLV, K_COEFF_VDW, K_COEFF_HBOND, K_COEFF_ESTAT, K_COEFF_DESOLV, K_COEFF_TORS
};

// gpfparser.cpp:34-175: first white-space token, case-insensitive exact match.
Kw classify_gpf(const char *line)
{
    while (*line && std::isspace((unsigned char)*line)) line++;
    char w[256];
    int i = 0;
    while (line[i] && !std::isspace((unsigned char)line[i]) && i < 255) { w[i] = line[i]; i++; }
    w[i] = 0;
    if (w[0] == 0) return K_NULL;
    if (w[0] == '#') return K_COMMENT;
    static const struct { const char *s; Kw k; } tab[] = {
        {"receptor_types", K_RECEPTOR_TYPES}, {"receptor", K_RECEPTOR}, {"gridfld", K_GRIDFLD},
        {"npts", K_NPTS}, {"spacing", K_SPACING}, {"gridcenter", K_GRIDCENTER},
        {"types", K_LIGAND_TYPES}, {"ligand_types", K_LIGAND_TYPES}, {"map", K_MAP},
        {"elecmap", K_ELECMAP}, {"dsolvmap", K_DSOLVMAP}, {"desolvmap", K_DSOLVMAP},
        {"covalentmap", K_COVALENTMAP}, {"coeff_vdw", K_COEFF_VDW}, {"coeff_hbond", K_COEFF_HBOND},
        {"coeff_estat", K_COEFF_ESTAT}, {"coeff_desolv", K_COEFF_DESOLV}, {"coeff_tors", K_COEFF_TORS},
        {"nbp_coeffs", K_NBP_COEFFS}, {"nbp_r_eps", K_NBP_R_EPS}, {"dielectric", K_DIEL},
        {"qasp", K_QASP}, {"fmap", K_FMAP}, {"disorder_h", K_DISORDER}, {"smooth", K_SMOOTH},
        {"sol_par", K_SOL_PAR}, {"constant", K_CONSTANT}, {"parameter_file", K_PARAM_FILE},
        {"use_vina_potential", K_USE_VINA}, {"outlev", K_OUTLEV},
        {"map_receptor_interior", K_MAP_RECEPTOR_INTERIOR}, {"cmap", K_CMAP},
        {"constriction_map", K_CMAP}, {"constriction_distance_cutoff", K_CONSTRICTION_CUTOFF},
        {"separate_desolvation_maps", K_SEPARATE_DESOLV}};
    for (auto &e : tab)
        if (strcasecmp(w, e.s) == 0) return e.k;
    return K_UNKNOWN;
}

// parsetypes.cpp:31-99: white-space separated words after the keyword.
std::vector<std::string> parse_types(const char *line)
{
    std::vector<std::string> out;
    const char *p = line;
    bool kw = false;
    while (*p) {
        while (*p && std::isspace((unsigned char)*p)) p++;
        if (!*p) break;
        const char *s = p;
        while (*p && !std::isspace((unsigned char)*p)) p++;
        if (!kw) { kw = true; continue; }
        out.emplace_back(s, (size_t)(p - s));
        if ((int)out.size() >= AG_MAX_MAPS - 2) break;  // MAX_ATOM_TYPES (autocomm.h:93)
    }
    return out;
}

// distdepdiel.cpp:30-57, Mehler & Solmajer distance-dependent dielectric.
double ddd_mehler_solmajer(double distance, double approx_zero)
{
    const double lambda = 0.003627, epsilon0 = 78.4, A = -8.5525, rk = 7.7839;
    const double B = epsilon0 - A;
    const double lambda_B = -lambda * B;
    double epsilon = A + B / (1.0 + rk * std::exp(lambda_B * distance));
    if (epsilon < approx_zero) epsilon = 1.0;
    return epsilon;
}

inline double angstrom(int i) { return ((double)i) * (1. / AG_A_DIV); }  // autogrid.h:88

// vect3len, main.cpp:98: nested hypot.
inline double vlen(const double v[3]) { return std::hypot(v[0], std::hypot(v[1], v[2])); }

// main.cpp:3606-3616
double vect_normalize(double v[3])
{
    double rd = vlen(v);
    double inv = (rd < kApproxZero) ? 1. / kApproxZero : 1. / rd;
    for (int i = 0; i < 3; i++) v[i] *= inv;
    return rd;
}

// main.cpp:3619-3633
double vect_sub_normalize(double out[3], const double a[3], const double b[3])
{
    double rd2 = 0.;
    for (int i = 0; i < 3; i++) { out[i] = a[i] - b[i]; rd2 += out[i] * out[i]; }
    double rd = (rd2 < kApproxZero) ? kApproxZero : std::sqrt(rd2);
    double inv = 1. / rd;
    for (int i = 0; i < 3; i++) out[i] *= inv;
    return rd;
}

// distance_le macro, main.cpp:122-128: component pre-checks, then nested-hypot length.
bool distance_le(const double a[3], const double b[3], double limit, double dc[3], double &d)
{
    for (int i = 0; i < 3; i++) {
        dc[i] = a[i] - b[i];
        if (!(dc[i] <= limit && dc[i] >= -limit)) return false;
    }
    d = vlen(dc);
    return d <= limit;
}

// Which neighbours define a directional atom's bond vectors (main.cpp:2320-2656).
struct BondRec {
    enum Kind { NONE = 0, D1, A2_ONE, A2_DIS, A2_TWO, A1 };
    int kind = NONE;
    int i1 = -1, i2 = -1;  // D1: parent; A2_ONE: bonded atom, its last neighbour; A2_DIS: carbon; A2_TWO: both
    int nb = 0, nbr[3] = {-1, -1, -1};  // A1: bonded atoms
};

struct MapObj {  // main.cpp:289-315
    int atom_type = 0, map_index = 0, is_covalent = 0, is_hbonder = 0;
    std::string filename, type;
    std::FILE *fp = nullptr;
    double vol_probe = 0, solpar_probe = 0, Rij = 0, epsij = 0, Rij_hb = 0, epsij_hb = 0;
    int hbond = 0;
    double cA[AG_MAX_REC_TYPES] = {}, cB[AG_MAX_REC_TYPES] = {};
    double nbp_r[AG_MAX_REC_TYPES] = {}, nbp_eps[AG_MAX_REC_TYPES] = {};
    int xA[AG_MAX_REC_TYPES] = {}, xB[AG_MAX_REC_TYPES] = {}, hbonder[AG_MAX_REC_TYPES] = {};
    double emin = kBig, emax = -kBig;
};

std::string fmt(const char *f, ...)
{
    char buf[2048];
    va_list ap;
    va_start(ap, f);
    std::vsnprintf(buf, sizeof buf, f, ap);
    va_end(ap);
    return buf;
}

}  // namespace

struct Job {
    // files and logging
    std::string gpf_path, receptor_filename, fld_filename, xyz_filename;
    std::FILE *glg = nullptr;
    bool glg_owned = false;
    std::FILE *fld_fp = nullptr, *xyz_fp = nullptr;
    clock_t t_start = 0;

    ParamLibrary lib;
    FEModel ad4;
    int outlev = 1;

    // receptor (main.cpp:360-379)
    int n_atoms = 0;
    std::vector<double> coord, charge, vol, solpar, rvector, rvector2;
    std::vector<int32_t> atom_type, hbond, rexp;
    std::vector<uint8_t> disorder;
    std::vector<int> nbonds;
    std::vector<std::array<int, kMaxNBonds>> bonded;
    std::vector<BondRec> bondrec;
    // ag_job_table_params: [map][type] parameter arrays
    std::vector<double> tp_cA, tp_cB, tp_R, tp_eps;
    std::vector<int32_t> tp_xA, tp_xB, tp_cov;
    std::vector<std::string> receptor_types;  // by rec index
    int receptor_types_ct = 0, receptor_types_gpf_ct = 0;
    bool has_receptor_types_in_gpf = false;
    std::vector<int> receptor_type_count;
    double q_max = -kBig, q_min = kBig, q_tot = 0;
    double cmax[3] = {-kBig, -kBig, -kBig}, cmin[3] = {kBig, kBig, kBig}, csum[3] = {0, 0, 0};
    double cmean[3] = {0, 0, 0};

    // grid
    int nelements[3] = {0, 0, 0}, n1[3] = {0, 0, 0}, ne[3] = {0, 0, 0};
    long long num_grid_points_per_map = -1;
    double spacing = 0.375, center[3] = {0, 0, 0}, cext[3], cgridmin[3], cgridmax[3];

    // maps
    std::vector<std::string> ligand_types;  // one per atom map
    int num_atom_maps = 0, num_maps = 0, elecPE = -1, dsolvPE = -1;
    bool gridmap_allocated = false;
    std::vector<MapObj> gridmap;
    bool separate_desolvation_maps = false;
    bool floating_grid = false, constriction_grid = false;
    std::string floating_filename, constriction_filename;
    std::FILE *floating_fp = nullptr, *constriction_fp = nullptr;
    double constriction_cutoff = 7.5;
    // The reference's default build never tests collisions (main.cpp:2893-2927
    // is compiled out); its USE_BHTREE build tests them unless the GPF says
    // "map_receptor_interior on" (main.cpp:580).  This front end keeps the
    // default build's behaviour unless the GPF says "off".
    bool map_receptor_interior = true;

    // physics switches
    double covpos[3] = {0, 0, 0}, covhalfwidth = 1.0, covbarrier = 1000.0;
    bool disorder_h = false, dddiel = false;
    double r_smooth = 0.5, solpar_q = 0.01097, diel = 0, invdielcal = 0;
    std::vector<double> epsilon_fn, r_epsilon_fn, sol_fn;
    std::vector<float> e_vdw_hb;  // [rec_types][atom_maps][NEINT]
    int hydrogen = -1, nonHB_hydrogen = -1, carbon = -1, arom_carbon = -1, oxygen = -1,
        nitrogen = -1, nonHB_nitrogen = -1, sulphur = -1, nonHB_sulphur = -1;

    // flat views handed to the hot path
    std::vector<int32_t> m_is_cov, m_is_hb, m_hbond;
    std::vector<double> m_solpar, m_vol;
    ag_problem prob{};
    // Vina-potential image of the same job (built on request)
    std::vector<float> vina_tab;
    std::vector<int32_t> vina_is_hb;
    std::vector<double> vina_zero;
    ag_problem vina_prob{};
    bool vina_built = false;
    bool finished = false;

    ~Job()
    {
        for (auto &m : gridmap)
            if (m.fp) std::fclose(m.fp);
        if (fld_fp) std::fclose(fld_fp);
        if (xyz_fp) std::fclose(xyz_fp);
        if (floating_fp) std::fclose(floating_fp);
        if (constriction_fp) std::fclose(constriction_fp);
        if (glg && glg_owned) std::fclose(glg);
    }

    void log(const std::string &s)
    {
        if (glg) { std::fputs(s.c_str(), glg); std::fflush(glg); }
    }
    void warn(const std::string &s) { log(fmt("\n%s: WARNING:  %s\n\n", kProgram, s.c_str())); }
    [[noreturn]] void fatal(const std::string &s, ag_status st = AG_ERR_FATAL_INPUT)
    {
        throw Fatal(st, s);
    }
    int rec_index(const std::string &t)
    {
        ParamEntry *e = lib.find(t);
        return e ? e->rec_index : -1;
    }
    int map_index(const std::string &t)
    {
        ParamEntry *e = lib.find(t);
        return e ? e->map_index : -1;
    }
    void set_canned_types()  // main.cpp:1415-1427, :2284-2292
    {
        hydrogen = rec_index("HD");
        nonHB_hydrogen = rec_index("H");
        carbon = rec_index("C");
        arom_carbon = rec_index("A");
        oxygen = rec_index("OA");
        nitrogen = rec_index("NA");
        nonHB_nitrogen = rec_index("N");
        sulphur = rec_index("SA");
        nonHB_sulphur = rec_index("S");
    }
    std::FILE *open_w(const std::string &name, const std::string &what)
    {
        std::FILE *f = std::fopen(name.c_str(), "w");
        if (!f) fatal("can't open file \"" + name + "\" for writing " + what + ".", AG_ERR_IO);
        return f;
    }

    void load(const std::string &gpf);
    void read_receptor(const char *line);
    void kw_ligand_types(const char *line);
    void kw_nbp(const char *line, bool r_eps);
    void kw_dielectric(const char *line);
    void finish_setup();
    void build_tables();
    void build_bond_vectors();
    void eval_bond_vectors(const double *xyz, double *rv, double *rv2) const;
    void bond_vectors_backward(const double *xyz, const double *g_rv, const double *g_rv2, double *g_xyz) const;
    void build_disorder();
    void make_problem();
    void build_vina_problem();
    void write_maps(const double *maps64, const float *maps32);
    void write_text(const char *text, const size_t *bytes, const double *emin, const double *emax);
};

// ---------------------------------------------------------------- receptor --
// main.cpp:823-1047
void Job::read_receptor(const char *gpf_line)
{
    char name[1024] = {0};
    std::sscanf(gpf_line, "%*s %1023s", name);
    receptor_filename = name;
    if (receptor_filename.empty()) fatal("No name specified for receptor filename");
    log(fmt("\nReceptor Input File :\t%s\n\n", name));
    std::FILE *f = std::fopen(name, "r");
    if (!f) fatal(fmt("can't find or open receptor PDBQT file \"%s\".", name), AG_ERR_IO);
    char line[1024];
    int lc = 0;
    std::string last_type;  // sscanf("%s") leaves the previous value on failure
    while (std::fgets(line, sizeof line, f)) {
        lc++;
        if (!(std::strncmp(line, "ATOM  ", 6) == 0 || std::strncmp(line, "HETATM", 6) == 0 ||
              std::strncmp(line, "CHAR", 4) == 0))
            continue;
        if (n_atoms >= AG_MAX_ATOMS) {
            std::fclose(f);
            fatal(fmt("Too many atoms in receptor PDBQT file %s line %d; the maximum is %d", name, lc,
                      AG_MAX_ATOMS), AG_ERR_TOO_LARGE);
        }
        if (std::strlen(line) < 78) {
            std::fclose(f);
            fatal(fmt("ATOM/HETATM line is too short in receptor PDBQT file %s line %d;", name, lc));
        }
        char f1[9], f2[9], f3[9], fq[7], ft[3];
        std::memcpy(f1, line + 30, 8); f1[8] = 0;
        std::memcpy(f2, line + 38, 8); f2[8] = 0;
        std::memcpy(f3, line + 46, 8); f3[8] = 0;
        double x = 0, y = 0, z = 0;
        if (std::sscanf(f1, "%lf", &x) + std::sscanf(f2, "%lf", &y) + std::sscanf(f3, "%lf", &z) != 3) {
            std::fclose(f);
            fatal(fmt("ATOM/HETATM line bad x,y,z in receptor PDBQT file %s line %d;", name, lc));
        }
        std::memcpy(fq, line + 70, 6); fq[6] = 0;
        double q = 0;
        std::sscanf(fq, "%lf", &q);
        ft[0] = line[77]; ft[1] = line[78]; ft[2] = 0;
        char tb[8];
        if (std::sscanf(ft, "%7s", tb) == 1) last_type = tb;
        ParamEntry *pe = lib.find(last_type);
        if (!pe) {
            std::fclose(f);
            fatal(fmt("receptor file contains unknown type: '%s line %d'\nadd parameters for it to the "
                      "parameter library first", last_type.c_str(), lc));
        }
        if (pe->rec_index < 0) {
            if (receptor_types_ct >= AG_MAX_REC_TYPES) {
                std::fclose(f);
                fatal("too many receptor atom types", AG_ERR_TOO_LARGE);
            }
            if ((int)receptor_types.size() <= receptor_types_ct) receptor_types.resize(receptor_types_ct + 1);
            receptor_types[receptor_types_ct] = pe->type;
            pe->rec_index = receptor_types_ct++;
        }
        coord.push_back(x); coord.push_back(y); coord.push_back(z);
        charge.push_back(q);
        atom_type.push_back(pe->rec_index);
        solpar.push_back(pe->solpar);
        vol.push_back(pe->vol);
        hbond.push_back(pe->hbond);
        if ((int)receptor_type_count.size() <= pe->rec_index) receptor_type_count.resize(pe->rec_index + 1);
        receptor_type_count[pe->rec_index]++;
        q_max = std::max(q_max, q);
        q_min = std::min(q_min, q);
        const double c3[3] = {x, y, z};
        for (int i = 0; i < 3; i++) {
            cmax[i] = std::max(cmax[i], c3[i]);
            cmin[i] = std::min(cmin[i], c3[i]);
            csum[i] += c3[i];
        }
        q_tot += q;
        n_atoms++;
    }
    std::fclose(f);
    if (has_receptor_types_in_gpf && receptor_types_ct != receptor_types_gpf_ct)
        fatal(fmt("The number of atom types found in the receptor PDBQT (%d) does not match the number "
                  "specified by the \"receptor_types\" command (%d) in the GPF!",
                  receptor_types_ct, receptor_types_gpf_ct));
    log(fmt("\nMaximum partial atomic charge found = %+.3lf e\n", q_max));
    log(fmt("Minimum partial atomic charge found = %+.3lf e\n\n", q_min));
    if (q_max == 0. && q_min == 0.)
        fatal(fmt("No partial atomic charges were found in the receptor PDBQT file %s!", name));
    rexp.assign(n_atoms, 0);
    log(fmt("\nTotal number of atoms :\t\t%d atoms \n", n_atoms));
    log(fmt("Total charge :\t\t\t%.2lf e\n", q_tot));
    for (int i = 0; i < 3; i++) cmean[i] = csum[i] / (double)n_atoms;
}

// ------------------------------------------------------------ ligand types --
// main.cpp:1170-1381
void Job::kw_ligand_types(const char *line)
{
    if (n1[0] == 0) fatal("You need to set the \"npts\" before setting the ligand types\".");
    std::vector<std::string> types = parse_types(line);
    for (const std::string &t : types) {
        ligand_types.push_back(t);
        num_atom_maps++;
        if (t != "Z" && separate_desolvation_maps) {
            ligand_types.push_back(t);
            num_atom_maps++;
        }
    }
    if (num_atom_maps > AG_MAX_MAPS - 2) fatal("too many ligand atom maps", AG_ERR_TOO_LARGE);
    for (int i = 0; i < num_atom_maps; i++) {
        ParamEntry *pe = lib.find(ligand_types[i]);
        if (!pe)
            fatal(fmt("unknown ligand atom type %s\nadd parameters for it to the parameter library first!",
                      ligand_types[i].c_str()));
        pe->map_index = i;
    }
    gridmap.assign(num_atom_maps + 2, MapObj());
    gridmap_allocated = true;
    log(fmt("Allocated space for %d gridmap objects\n", num_atom_maps + 2));
    if (num_grid_points_per_map < 0)
        fatal("You need to set the number of grid points using \"npts\" before setting the ligand atom types.");
    for (int i = 0; i < num_atom_maps; i++) {
        MapObj &g = gridmap[i];
        g.map_index = i;
        g.type = ligand_types[i];
        ParamEntry *pe = lib.find(ligand_types[i]);
        if (ligand_types[i] == "Z") g.is_covalent = 1;
        g.atom_type = pe->map_index;
        g.solpar_probe = pe->solpar;
        g.vol_probe = pe->vol;
        g.Rij = pe->Rij;
        g.epsij = pe->epsij_unweighted * ad4.coeff_vdW;
        g.hbond = pe->hbond;
        g.Rij_hb = pe->Rij_hb;
        g.epsij_hb = pe->epsij_hb_unweighted * ad4.coeff_hbond;
        if (g.hbond > 0) g.is_hbonder = 1;
        for (int j = 0; j < receptor_types_ct; j++) {
            ParamEntry *rp = lib.find(receptor_types[j]);
            if (!rp) continue;
            g.nbp_r[j] = (g.Rij + rp->Rij) / 2.;
            g.nbp_eps[j] = std::sqrt(g.epsij * rp->epsij_unweighted * ad4.coeff_vdW);
            g.xA[j] = 12;
            g.xB[j] = 6;
            g.hbonder[j] = 0;
            const int rh = rp->hbond;
            if ((g.hbond > 2 || g.hbond == 6) && (rh == 1 || rh == 2 || rh == 6)) {
                g.xB[j] = 10; g.hbonder[j] = 1; g.is_hbonder = 1;
                g.nbp_r[j] = g.Rij_hb;
                g.nbp_eps[j] = g.epsij_hb;
            } else if ((g.hbond == 1 || g.hbond == 2 || g.hbond == 6) && rh > 2) {
                g.xB[j] = 10; g.hbonder[j] = 1; g.is_hbonder = 1;
                g.nbp_r[j] = rp->Rij_hb;
                g.nbp_eps[j] = rp->epsij_hb_unweighted * ad4.coeff_hbond;
            }
        }
    }
}

// ----------------------------------------------------- nbp_r_eps/nbp_coeffs --
// main.cpp:1741-1806
void Job::kw_nbp(const char *line, bool r_eps)
{
    double Rij = 0, epsij = 0, cA = 0, cB = 0;
    int xA = 0, xB = 0;
    char p0[256] = {0}, p1[256] = {0};
    int nf = std::sscanf(line, "%*s %lf %lf %d %d %255s %255s", &Rij, &epsij, &xA, &xB, p0, p1);
    if (nf != 6) fatal("syntax error, not 6 values in NBP_R_EPS line");
    if (r_eps) {
        epsij *= ad4.coeff_vdW;
        if (xA != xB) {
            double tmpconst = epsij / (double)(xA - xB);
            cA = tmpconst * std::pow(Rij, (double)xA) * (double)xB;
            cB = tmpconst * std::pow(Rij, (double)xB) * (double)xA;
        } else {
            fatal("exponents xA and xB cannot be equal.");
        }
    } else {
        cA = Rij;
        cB = epsij;
    }
    const char *param[2] = {p0, p1};
    for (int i = 0; i < 2; i++) {
        int lig = map_index(param[i % 2]);
        int rec = rec_index(param[(i + 1) % 2]);
        if (lig >= 0 && rec >= 0) {
            if (!gridmap_allocated || lig >= (int)gridmap.size() || rec >= AG_MAX_REC_TYPES)
                fatal("nbp_r_eps/nbp_coeffs before ligand_types");
            MapObj &g = gridmap[lig];
            g.cA[rec] = cA; g.cB[rec] = cB;
            g.nbp_r[rec] = Rij; g.nbp_eps[rec] = epsij;
            g.xA[rec] = xA; g.xB[rec] = xB;
        }
    }
}

// -------------------------------------------------------------- dielectric --
// main.cpp:1607-1639
void Job::kw_dielectric(const char *line)
{
    std::sscanf(line, "%*s %lf", &diel);
    if (diel < 0.) {
        dddiel = true;
        epsilon_fn.assign(AG_NDIEL, 0.0);
        r_epsilon_fn.assign(AG_NDIEL, 0.0);
        epsilon_fn[0] = 1.0;
        for (int i = 1; i < AG_NDIEL; i++) epsilon_fn[i] = ddd_mehler_solmajer(angstrom(i), kApproxZero);
        for (int i = 0; i < AG_NDIEL; i++) r_epsilon_fn[i] = kFactor / epsilon_fn[i];
        log("\nUsing *distance-dependent* dielectric function of Mehler and Solmajer, Prot.Eng.4, 903-910.\n\n");
    } else {
        dddiel = false;
        if (diel <= kApproxZero) diel = 40.;
        log(fmt("Using a *constant* dielectric of:  %.2f\n", diel));
        invdielcal = kFactor / diel;
    }
}

// ------------------------------------------------------------------- load --
void Job::load(const std::string &gpf)
{
    gpf_path = gpf;
    std::FILE *g = std::fopen(gpf.c_str(), "r");
    if (!g) fatal("Sorry, I can't find or open Grid Parameter File \"" + gpf + "\"", AG_ERR_IO);
    std::unique_ptr<std::FILE, int (*)(std::FILE *)> gcloser(g, std::fclose);
    lib.load_defaults(ad4);  // main.cpp:771
    r_epsilon_fn.assign(AG_NDIEL, 0.0);
    char raw[1024];
    while (std::fgets(raw, sizeof raw, g)) {
        Kw kw = classify_gpf(raw);
        log(std::string("GPF> ") + raw);
        if (kw == K_UNKNOWN) {
            warn("Unrecognized keyword in grid parameter file.");
            continue;
        }
        char line[1024];
        std::strcpy(line, raw);
        if (kw != K_NULL && kw != K_COMMENT) {
            char *hash = std::strchr(line, '#');  // strindex(GPF_line, "#") truncation
            if (hash) *hash = 0;
        }
        switch (kw) {
            case K_NULL: case K_COMMENT: break;
            case K_RECEPTOR: read_receptor(line); break;
            case K_GRIDFLD: {  // main.cpp:1051-1079
                char name[1024] = {0};
                std::sscanf(line, "%*s %1023s", name);
                fld_filename = name;
                if (fld_filename.empty()) fatal("No name specified for AVS_fld_filename");
                size_t pos = fld_filename.find(".fld");
                if (pos == std::string::npos) fatal("Grid data file needs the extension \".fld\" for AVS input");
                size_t f = fld_filename.find("fld");
                xyz_filename = fld_filename;
                xyz_filename.replace(f, 3, "xyz");
                fld_fp = open_w(fld_filename, "grid dimensions data file");
                xyz_fp = open_w(xyz_filename, "grid extrema data file");
            } break;
            case K_NPTS: {  // main.cpp:1083-1105, check_size.cpp:36-83
                std::sscanf(line, "%*s %d %d %d", &nelements[0], &nelements[1], &nelements[2]);
                for (int i = 0; i < 3; i++) {
                    if (nelements[i] < 0) fatal(fmt("Negative number of %c-grid elements!", "xyz"[i]));
                    if (nelements[i] == 0) fatal(fmt("0 %c-grid elements!", "xyz"[i]));
                    if (nelements[i] > AG_MAX_GRID_PTS)
                        fatal(fmt("Maximum number of %c-grid elements allowed is %d.", "xyz"[i], AG_MAX_GRID_PTS));
                    nelements[i] = (nelements[i] / 2) * 2;
                    ne[i] = nelements[i] / 2;
                    n1[i] = nelements[i] + 1;
                }
                num_grid_points_per_map = (long long)n1[0] * n1[1] * n1[2];
                log(fmt("\nNumber of grid points in x-direction:\t%d\n", n1[0]));
                log(fmt("Number of grid points in y-direction:\t%d\n", n1[1]));
                log(fmt("Number of grid points in z-direction:\t%d\n\n", n1[2]));
            } break;
            case K_SPACING: std::sscanf(line, "%*s %lf", &spacing); break;
            case K_GRIDCENTER: {  // main.cpp:1117-1166
                if (!fld_fp || !xyz_fp)
                    fatal("You need to set the \"gridfld\" file before setting the grid center\".");
                char tok[256] = {0};
                std::sscanf(line, "%*s %255s", tok);
                if (std::strncmp(tok, "auto", 4) == 0) {
                    for (int i = 0; i < 3; i++) center[i] = cmean[i];
                } else {
                    std::sscanf(line, "%*s %lf %lf %lf", &center[0], &center[1], &center[2]);
                }
                for (int ia = 0; ia < n_atoms; ia++)
                    for (int i = 0; i < 3; i++) coord[3 * ia + i] -= center[i];
                for (int i = 0; i < 3; i++) {
                    cext[i] = spacing * (double)ne[i];
                    cgridmax[i] = center[i] + cext[i];
                    cgridmin[i] = center[i] - cext[i];
                }
                for (int i = 0; i < 3; i++) std::fprintf(xyz_fp, "%.3lf %.3lf\n", cgridmin[i], cgridmax[i]);
                std::fclose(xyz_fp);
                xyz_fp = nullptr;
            } break;
            case K_LIGAND_TYPES: kw_ligand_types(line); break;
            case K_RECEPTOR_TYPES: {  // main.cpp:1385-1431
                std::vector<std::string> t = parse_types(line);
                if ((int)t.size() > AG_MAX_REC_TYPES) fatal("too many receptor types", AG_ERR_TOO_LARGE);
                receptor_types_ct = (int)t.size();
                receptor_types_gpf_ct = receptor_types_ct;
                has_receptor_types_in_gpf = true;
                receptor_types = t;
                for (int i = 0; i < receptor_types_ct; i++) {
                    ParamEntry *pe = lib.find(t[i]);
                    if (!pe)
                        fatal("Unknown receptor type: \"" + t[i] +
                              "\"\n -- Add parameters for it to the parameter library first!");
                    pe->rec_index = i;
                }
                set_canned_types();
            } break;
            case K_SOL_PAR: {  // main.cpp:1435-1456
                char t[64] = {0};
                double v = 0, s = 0;
                std::sscanf(line, "%*s %63s %lf %lf", t, &v, &s);
                ParamEntry *pe = lib.find(t);
                if (pe) {
                    pe->vol = v;
                    pe->solpar = s;
                    if (pe->map_index >= 0 && pe->map_index < (int)gridmap.size())
                        gridmap[pe->map_index].solpar_probe = s;
                } else {
                    log(fmt("%s key not found\n", t));
                }
            } break;
            case K_USE_VINA: fatal("Vina potential not implemented", AG_ERR_UNSUPPORTED);
            case K_MAP: {  // main.cpp:1475-1502
                if (!gridmap_allocated) fatal("\"map\" keyword before \"ligand_types\"");
                if (num_maps > num_atom_maps + (elecPE > -1 ? 1 : 0) + (dsolvPE > -1 ? 1 : 0))
                    fatal(fmt("Too many \"map\" keywords (%d);  the \"ligand_types\" command declares only %d "
                              "atom types.\nRemove a \"map\" keyword from the GPF.", num_maps, num_atom_maps));
                if (num_maps >= (int)gridmap.size())  // the reference writes past gridmap[] here
                    fatal(fmt("Too many map requests (%d) for %d declared atom types", num_maps + 1, num_atom_maps));
                char name[1024] = {0};
                std::sscanf(line, "%*s %1023s", name);
                if (!name[0]) fatal("No name specified for map file");
                gridmap[num_maps].filename = name;
                gridmap[num_maps].fp = open_w(name, "grid map");
                log(fmt("\nOutput Grid Map %d:   %s\n\n", num_maps + 1, name));
                num_maps++;
            } break;
            case K_ELECMAP: case K_DSOLVMAP: {  // main.cpp:1505-1544
                const bool e = (kw == K_ELECMAP);
                int &pe = e ? elecPE : dsolvPE;
                if (pe >= 0) fatal(e ? "Duplicate \"elecmap\" request" : "Duplicate \"dsolvmap\" request");
                if (num_maps < num_atom_maps)
                    fatal(e ? "\"elecmap\" request appeared before all atom map requests had appeared."
                            : "\"desolvmap\" request appeared before all atom map requests had appeared.");
                if (!gridmap_allocated || num_maps >= (int)gridmap.size())
                    fatal(fmt("Too many map requests (%d) for %d declared atom types", num_maps + 1, num_atom_maps));
                pe = num_maps;
                char name[1024] = {0};
                std::sscanf(line, "%*s %1023s", name);
                if (!name[0])
                    fatal(e ? "No name specified for electrostatic map" : "No name specified for desolvation map");
                gridmap[pe].filename = name;
                gridmap[pe].fp = open_w(name, e ? "electrostatic map" : "desolvation map");
                num_maps++;
            } break;
            case K_COVALENTMAP:  // main.cpp:1547-1557
                std::sscanf(line, "%*s %lf %lf %lf %lf %lf", &covhalfwidth, &covbarrier, &covpos[0], &covpos[1],
                            &covpos[2]);
                for (int i = 0; i < 3; i++) covpos[i] -= center[i];
                break;
            case K_DISORDER: disorder_h = true; break;
            case K_SMOOTH: std::sscanf(line, "%*s %lf", &r_smooth); break;
            case K_CONSTRICTION_CUTOFF: std::sscanf(line, "%*s %lf", &constriction_cutoff); break;
            case K_SEPARATE_DESOLV:
                if (num_atom_maps > 0) fatal("\"separate_desolvation_maps\" must be specified before \"ligand_types\"");
                separate_desolvation_maps = true;
                break;
            case K_OUTLEV: std::sscanf(line, "%*s %d", &outlev); break;
            case K_QASP: std::sscanf(line, "%*s %lf", &solpar_q); break;
            case K_DIEL: kw_dielectric(line); break;
            case K_MAP_RECEPTOR_INTERIOR: {  // main.cpp:1642-1659
                char tok[64] = "true";
                std::sscanf(line, "%*s %63s", tok);
                // the reference's USE_BHTREE build accepts "off" (collisions
                // reported); its default build stops with a fatal error there.
                // This front end takes the USE_BHTREE behaviour.
                if (strcasecmp(tok, "true") == 0 || strcasecmp(tok, "on") == 0) {
                    map_receptor_interior = true;
                    log("Mapping receptor interior instead of reporting collision if nearer than 1.50 to any atom.");
                } else {
                    map_receptor_interior = false;
                    log("Reporting collision if nearer than 1.50 to any atom.");
                }
            } break;
            case K_FMAP: case K_CMAP: {  // main.cpp:1663-1695
                const bool fm = (kw == K_FMAP);
                if (fm ? floating_grid : constriction_grid)
                    fatal(fm ? "Muliple requests for floating map are not allowed."
                             : "Muliple requests for constriction map are not allowed.");
                char name[1024] = {0};
                std::sscanf(line, "%*s %1023s", name);
                if (!name[0]) fatal(fm ? "No name specified for floating map" : "No name specified for constriction map");
                if (fm) { floating_filename = name; floating_fp = open_w(name, "floating map"); floating_grid = true; }
                else { constriction_filename = name; constriction_fp = open_w(name, "constriction map"); constriction_grid = true; }
            } break;
            case K_COEFF_VDW: std::sscanf(line, "%*s %lf", &ad4.coeff_vdW); break;
            case K_COEFF_HBOND: std::sscanf(line, "%*s %lf", &ad4.coeff_hbond); break;
            case K_COEFF_ESTAT: std::sscanf(line, "%*s %lf", &ad4.coeff_estat); break;
            case K_COEFF_DESOLV: std::sscanf(line, "%*s %lf", &ad4.coeff_desolv); break;
            case K_COEFF_TORS: std::sscanf(line, "%*s %lf", &ad4.coeff_tors); break;
            case K_PARAM_FILE: {  // main.cpp:1726-1736
                char name[1024] = {0};
                std::sscanf(line, "%*s %1023s", name);
                if (!name[0]) fatal("No name specified for FN_parameter_library");
                lib.load_file(name, ad4);
            } break;
            case K_NBP_COEFFS: kw_nbp(line, false); break;
            case K_NBP_R_EPS: kw_nbp(line, true); break;
            default: break;
        }
    }
    finish_setup();
}

// ------------------------------------------------ after the GPF: checks, fld --
// main.cpp:1848-1956
void Job::finish_setup()
{
    if (num_atom_maps > (num_maps - (elecPE >= 0 ? 1 : 0) - (dsolvPE >= 0 ? 1 : 0)))
        fatal("Too few \"map\" keywords found for the number of ligand atom types.");
    if (elecPE < 0) log("\nThe electrostatic map file is not defined in the GPF.\n");
    if (dsolvPE < 0) log("\nThe desolvation map file is not defined in the GPF.\n");
    if (!fld_fp) fatal("Missing \"gridfld\" keyword.");
    if (num_grid_points_per_map < 0) fatal("You need to set the number of grid points using \"npts\".");
    const int num_distance_maps = (floating_grid ? 1 : 0) + (constriction_grid ? 1 : 0);
    std::FILE *f = fld_fp;
    std::fprintf(f, "# AVS field file\n#\n");
    std::fprintf(f, "# AutoDock Atomic Affinity and Electrostatic Grids\n#\n");
    std::fprintf(f, "# Created by %s %s.\n#\n", kProgram, "4.2.7.x");
    std::fprintf(f, "#SPACING %.3f\n", (float)spacing);
    std::fprintf(f, "#NELEMENTS %d %d %d\n", nelements[0], nelements[1], nelements[2]);
    std::fprintf(f, "#CENTER %.3lf %.3lf %.3lf\n", center[0], center[1], center[2]);
    std::fprintf(f, "#MACROMOLECULE %s\n", receptor_filename.c_str());
    std::fprintf(f, "#GRID_PARAMETER_FILE %s\n#\n", gpf_path.c_str());
    std::fprintf(f, "ndim=3\t\t\t# number of dimensions in the field\n");
    std::fprintf(f, "dim1=%d\t\t\t# number of x-elements\n", n1[0]);
    std::fprintf(f, "dim2=%d\t\t\t# number of y-elements\n", n1[1]);
    std::fprintf(f, "dim3=%d\t\t\t# number of z-elements\n", n1[2]);
    std::fprintf(f, "nspace=3\t\t# number of physical coordinates per point\n");
    std::fprintf(f, "veclen=%d\t\t# number of affinity values at each point\n", num_maps + num_distance_maps);
    std::fprintf(f, "data=float\t\t# data type (byte, integer, float, double)\n");
    std::fprintf(f, "field=uniform\t\t# field type (uniform, rectilinear, irregular)\n");
    for (int i = 0; i < 3; i++)
        std::fprintf(f, "coord %d file=%s filetype=ascii offset=%d\n", i + 1, xyz_filename.c_str(), i * 2);
    for (int i = 0; i < num_atom_maps; i++) {
        std::fprintf(f, "label=%s-affinity\t# component label for variable %d\n", gridmap[i].type.c_str(), i + 1);
        if (separate_desolvation_maps && !gridmap[i].is_covalent) {
            i++;
            std::fprintf(f, "label=%s-desolv\t# component label for variable %d\n", gridmap[i].type.c_str(), i + 1);
        }
    }
    if (elecPE >= 0) std::fprintf(f, "label=Electrostatics\t# component label for variable %d\n", elecPE + 1);
    if (dsolvPE >= 0) std::fprintf(f, "label=Desolvation\t# component label for variable %d\n", dsolvPE + 1);
    if (floating_grid)
        std::fprintf(f, "label=Floating_Grid\t# component label for variable %d\n",
                     num_atom_maps + (elecPE >= 0) + (dsolvPE >= 0) + 1);
    if (constriction_grid)
        std::fprintf(f, "label=Constriction_Grid\t# component label for variable %d\n",
                     num_atom_maps + (elecPE >= 0) + (dsolvPE >= 0) + (floating_grid ? 1 : 0) + 1);
    std::fprintf(f, "#\n# location of affinity grid files and how to read them\n#\n");
    for (int i = 0; i < num_atom_maps; i++)
        std::fprintf(f, "variable %d file=%s filetype=ascii skip=6\n", i + 1, gridmap[i].filename.c_str());
    if (elecPE >= 0)
        std::fprintf(f, "variable %d file=%s filetype=ascii skip=6\n", num_atom_maps + 1, gridmap[elecPE].filename.c_str());
    if (dsolvPE >= 0)
        std::fprintf(f, "variable %d file=%s filetype=ascii skip=6\n", num_atom_maps + ((elecPE >= 0) ? 2 : 1),
                     gridmap[dsolvPE].filename.c_str());
    if (floating_grid)
        std::fprintf(f, "variable %d file=%s filetype=ascii skip=6\n", num_maps + 1, floating_filename.c_str());
    if (constriction_grid)
        std::fprintf(f, "variable %d file=%s filetype=ascii skip=6\n", num_maps + (floating_grid ? 1 : 0) + 1,
                     constriction_filename.c_str());
    std::fclose(fld_fp);
    fld_fp = nullptr;

    build_tables();
    set_canned_types();
    build_bond_vectors();
    if (disorder_h) build_disorder();
    // map headers, main.cpp:2752-2776
    auto header = [&](std::FILE *mf) {
        std::fprintf(mf, "GRID_PARAMETER_FILE %s\n", gpf_path.c_str());
        std::fprintf(mf, "GRID_DATA_FILE %s\n", fld_filename.c_str());
        std::fprintf(mf, "MACROMOLECULE %s\n", receptor_filename.c_str());
        std::fprintf(mf, "SPACING %.3lf\n", spacing);
        std::fprintf(mf, "NELEMENTS %d %d %d\n", nelements[0], nelements[1], nelements[2]);
        std::fprintf(mf, "CENTER %.3lf %.3lf %.3lf\n", center[0], center[1], center[2]);
        std::fflush(mf);
    };
    for (int k = 0; k < num_maps; k++) header(gridmap[k].fp);
    if (floating_fp) header(floating_fp);
    if (constriction_fp) header(constriction_fp);
    log(fmt("Beginning grid calculations.\n\nCalculating %d grid%s over %lld element%s, around %d receptor atom%s.\n\n",
            num_maps + num_distance_maps, (num_maps + num_distance_maps) == 1 ? "" : "s",
            num_grid_points_per_map, num_grid_points_per_map == 1 ? "" : "s", n_atoms, n_atoms == 1 ? "" : "s"));
    make_problem();
}

// ------------------------------------------------------------------ tables --
// vdW/H-bond tables main.cpp:2040-2266, desolvation main.cpp:2268-2276
void Job::build_tables()
{
    const int nR = std::max(receptor_types_ct, 1);
    e_vdw_hb.assign((size_t)nR * std::max(num_atom_maps, 1) * AG_NEINT, 0.0f);
    std::vector<double> smooth(AG_NEINT);
    for (int ia = 0; ia < num_atom_maps; ia++) {
        MapObj &g = gridmap[ia];
        if (g.is_covalent) continue;
        for (int i = 0; i < receptor_types_ct; i++) {
            double cA = g.cA[i], cB = g.cB[i], Rij = g.nbp_r[i], epsij = g.nbp_eps[i];
            int xA = g.xA[i], xB = g.xB[i];
            float *tab = &e_vdw_hb[((size_t)i * num_atom_maps + ia) * AG_NEINT];
            if (cA == 0 && cB == 0) {
                double tmpconst = epsij / (double)(xA - xB);
                cA = tmpconst * std::pow(Rij, (double)xA) * (double)xB;
                cB = tmpconst * std::pow(Rij, (double)xB) * (double)xA;
            }
            if (std::isnan(cA)) fatal("Van der Waals coefficient cA is not a number.  AutoGrid must exit.");
            if (std::isnan(cB)) fatal("Van der Waals coefficient cB is not a number.  AutoGrid must exit.");
            if (xA == 0) fatal("Van der Waals exponent xA is 0.  AutoGrid must exit.");
            if (xB == 0) fatal("Van der Waals exponent xB is 0.  AutoGrid must exit.");
            for (int k = 1; k < AG_NEINT; k++) {
                double r = angstrom(k);
                double rA = std::pow(r, (double)xA), rB = std::pow(r, (double)xB);
                double v = cA / rA - cB / rB;
                tab[k] = (float)((kEintClamp < v) ? kEintClamp : v);
            }
            tab[0] = (float)kEintClamp;
            tab[AG_NEINT - 1] = 0.f;
            int i_smooth = (int)(r_smooth * AG_A_DIV / 2.);
            if (i_smooth > 0) {
                for (int k = 0; k < AG_NEINT; k++) {
                    double s = 100000.;
                    int lo = std::max(0, k - i_smooth), hi = std::min(AG_NEINT, k + i_smooth + 1);
                    for (int j = lo; j < hi; j++) s = (s < (double)tab[j]) ? s : (double)tab[j];
                    smooth[k] = s;
                }
                for (int k = 0; k < AG_NEINT; k++) tab[k] = (float)smooth[k];
            }
        }
    }
    sol_fn.assign(AG_NDIEL, 0.0);
    const double sigma = 3.6;
    for (int k = 1; k < AG_NDIEL; k++) {
        double r = angstrom(k);
        sol_fn[k] = ad4.coeff_desolv * std::exp(-(r * r) / (2. * (sigma * sigma)));
    }
}

// ----------------------------------------------------------- bond vectors --
// main.cpp:2297-2659.  Detection (which neighbours define each directional
// atom's bond vectors) is recorded as a BondRec; eval_bond_vectors() then
// computes rvector/rvector2 from coordinates, so the same topology can be
// re-evaluated and differentiated at other coordinates.
void Job::build_bond_vectors()
{
    rvector.assign((size_t)3 * n_atoms, 0.0);
    rvector2.assign((size_t)3 * n_atoms, 0.0);
    disorder.assign(n_atoms, 0);
    nbonds.assign(n_atoms, 0);
    bonded.assign(n_atoms, std::array<int, kMaxNBonds>{{0, 0, 0, 0}});
    bondrec.assign(n_atoms, BondRec{});
    auto C = [&](int a) { return &coord[3 * (size_t)a]; };
    auto add_bond = [&](int i, int j) {  // bondmanager.cpp:44-88
        if (nbonds[i] >= kMaxNBonds || nbonds[j] >= kMaxNBonds)
            fatal("could not add bond");
        bonded[i][nbonds[i]++] = j;
        bonded[j][nbonds[j]++] = i;
    };
    for (int ia = 0; ia < n_atoms; ia++) {
        const int from = std::max(ia - 20, 0), to = std::min(ia + 20, n_atoms - 1);
        BondRec &br = bondrec[ia];
        if (hbond[ia] == 2) {  // D1 donor hydrogen, main.cpp:2320-2414
            for (int ib = from; ib <= to; ib++) {
                if (ib == ia) continue;
                double d[3], rd;
                if (!distance_le(C(ia), C(ib), 1.378, d, rd)) continue;
                br.kind = BondRec::D1;  // the last bonded atom in the scan wins
                br.i1 = ib;
                if (vect_normalize(d) == 0.)
                    warn(fmt("While calculating an H-O or H-N bond vector...\nAttempt to divide by zero was just "
                             "prevented.\nAre the coordinates of atoms %d and %d the same?", ia + 1, ib + 1));
                if (atom_type[ib] == nitrogen) rexp[ia] = 2;
                else if (atom_type[ib] == oxygen || atom_type[ib] == sulphur) rexp[ia] = 4;
                else rexp[ia] = 2;
                if (disorder_h) add_bond(ia, ib);
            }
        } else if (hbond[ia] == 5) {  // A2 acceptor, main.cpp:2416-2594
            int nbond = 0, i1 = -1, i2 = -1;
            for (int ib = from; ib <= to; ib++) {
                if (ib == ia) continue;
                double dc[3], rd;
                const double lim = (atom_type[ib] == hydrogen || atom_type[ib] == nonHB_hydrogen) ? 1.3 : 1.9;
                if (!distance_le(C(ia), C(ib), lim, dc, rd)) continue;
                if (nbond == 2) warn(fmt("Found an H-bonding O atom with three bonded atoms, atom serial number %d", ia + 1));
                else if (nbond == 1) { nbond = 2; i2 = ib; }
                else if (nbond == 0) { nbond = 1; i1 = ib; }
            }
            if (nbond == 0)
                warn(fmt("Oxygen atom found with no bonded atoms, atom serial number %d, atom_type %d", ia + 1, atom_type[ia]));
            if (nbond == 1) {
                br.kind = BondRec::A2_ONE;
                br.i1 = i1;
                for (int j2 = from; j2 <= to; j2++) {
                    if (j2 == i1 || j2 == ia) continue;
                    double d[3], rdcx;
                    if (!distance_le(C(i1), C(j2), atom_type[j2] == hydrogen ? 1.3 : 1.7, d, rdcx)) continue;
                    br.i2 = j2;  // the last neighbour of i1 in the scan wins
                }
            } else if (nbond == 2) {
                if (disorder_h && (atom_type[i1] == hydrogen || atom_type[i2] == hydrogen) &&
                    atom_type[i1] != atom_type[i2]) {
                    int ib;
                    if (atom_type[i1] == carbon || atom_type[i1] == arom_carbon) ib = i1;
                    else if (atom_type[i2] == carbon || atom_type[i2] == arom_carbon) ib = i2;
                    else ib = i1;
                    add_bond(ia, ib);
                    br.kind = BondRec::A2_DIS;
                    br.i1 = ib;
                } else {
                    br.kind = BondRec::A2_TWO;
                    br.i1 = i1;
                    br.i2 = i2;
                }
            }
        } else if (hbond[ia] == 4) {  // A1 directional N acceptor, main.cpp:2596-2656
            br.kind = BondRec::A1;
            br.nb = 0;
            for (int ib = from; ib <= to; ib++) {
                if (ib == ia) continue;
                const double lim = (atom_type[ib] == hydrogen || atom_type[ib] == nonHB_hydrogen) ? 1.3 : 1.7;
                double dc[3], rd;
                if (!distance_le(C(ia), C(ib), lim, dc, rd)) continue;
                br.nbr[br.nb] = ib;
                if (++br.nb == 3) break;
            }
            if (br.nb == 0) warn(fmt("Nitrogen atom found with no bonded atoms, atom serial number %d", ia + 1));
        }
    }
    eval_bond_vectors(coord.data(), rvector.data(), rvector2.data());
}

// The vector arithmetic of main.cpp:2320-2656 on the recorded topology.
void Job::eval_bond_vectors(const double *xyz, double *rv_out, double *rv2_out) const
{
    auto C = [&](int a) { return &xyz[3 * (size_t)a]; };
    std::fill(rv_out, rv_out + 3 * (size_t)n_atoms, 0.0);
    std::fill(rv2_out, rv2_out + 3 * (size_t)n_atoms, 0.0);
    for (int ia = 0; ia < n_atoms; ia++) {
        const BondRec &br = bondrec[ia];
        double *rv = rv_out + 3 * (size_t)ia, *rv2 = rv2_out + 3 * (size_t)ia;
        switch (br.kind) {
            case BondRec::D1:
                for (int i = 0; i < 3; i++) rv[i] = C(ia)[i] - C(br.i1)[i];
                vect_normalize(rv);
                break;
            case BondRec::A2_ONE:
                vect_sub_normalize(rv, C(ia), C(br.i1));
                if (br.i2 >= 0) {
                    double d[3];
                    for (int i = 0; i < 3; i++) d[i] = C(br.i1)[i] - C(br.i2)[i];
                    vect_normalize(d);
                    rv2[0] = rv[1] * d[2] - rv[2] * d[1];
                    rv2[1] = rv[2] * d[0] - rv[0] * d[2];
                    rv2[2] = rv[0] * d[1] - rv[1] * d[0];
                    vect_normalize(rv2);
                }
                break;
            case BondRec::A2_DIS:
                vect_sub_normalize(rv, C(ia), C(br.i1));
                break;
            case BondRec::A2_TWO: {
                vect_sub_normalize(rv2, C(br.i2), C(br.i1));
                double rdot = 0.;
                for (int i = 0; i < 3; i++) rdot += (C(ia)[i] - C(br.i1)[i]) * rv2[i];
                for (int i = 0; i < 3; i++) rv[i] = C(ia)[i] - ((rdot * rv2[i]) + C(br.i1)[i]);
                vect_normalize(rv);
            } break;
            case BondRec::A1: {
                double mean[3] = {0, 0, 0};
                for (int b = 0; b < br.nb; b++)
                    for (int i = 0; i < 3; i++) mean[i] += (C(ia)[i] - C(br.nbr[b])[i]) / br.nb;
                vect_normalize(mean);
                for (int i = 0; i < 3; i++) rv[i] = -1 * mean[i];
            } break;
            default: break;
        }
    }
}

namespace {
// Adjoint of vect_normalize (sub = false) / vect_sub_normalize (sub = true) at
// input v: gv = J^T gy, with J = (I - y y^T)/|v| above the zero threshold and
// J = I/threshold below it.
void normalize_bwd(const double v[3], const double gy[3], double gv[3], bool sub)
{
    double rd;
    bool below;
    if (sub) {
        const double rd2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        below = rd2 < kApproxZero;
        rd = below ? kApproxZero : std::sqrt(rd2);
    } else {
        rd = vlen(v);
        below = rd < kApproxZero;
        if (below) rd = kApproxZero;
    }
    if (below) {
        for (int i = 0; i < 3; i++) gv[i] = gy[i] / rd;
        return;
    }
    const double y[3] = {v[0] / rd, v[1] / rd, v[2] / rd};
    const double yg = y[0] * gy[0] + y[1] * gy[1] + y[2] * gy[2];
    for (int i = 0; i < 3; i++) gv[i] = (gy[i] - y[i] * yg) / rd;
}

inline void cross(const double a[3], const double b[3], double o[3])
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
}  // namespace

// g_xyz += d(rvector, rvector2)/d(xyz)^T (g_rv, g_rv2), FP64, on the recorded topology.
void Job::bond_vectors_backward(const double *xyz, const double *g_rv, const double *g_rv2, double *g_xyz) const
{
    auto C = [&](int a) { return &xyz[3 * (size_t)a]; };
    auto add = [&](int a, const double g[3], double s) {
        for (int i = 0; i < 3; i++) g_xyz[3 * (size_t)a + i] += s * g[i];
    };
    for (int ia = 0; ia < n_atoms; ia++) {
        const BondRec &br = bondrec[ia];
        const double *grv = g_rv + 3 * (size_t)ia, *grv2 = g_rv2 + 3 * (size_t)ia;
        switch (br.kind) {
            case BondRec::D1: {
                double v[3], gv[3];
                for (int i = 0; i < 3; i++) v[i] = C(ia)[i] - C(br.i1)[i];
                normalize_bwd(v, grv, gv, false);
                add(ia, gv, 1.);
                add(br.i1, gv, -1.);
            } break;
            case BondRec::A2_ONE: {
                double u[3], rv[3], g_rv_t[3] = {grv[0], grv[1], grv[2]};
                for (int i = 0; i < 3; i++) u[i] = C(ia)[i] - C(br.i1)[i];
                vect_sub_normalize(rv, C(ia), C(br.i1));
                if (br.i2 >= 0) {
                    double dd[3], dn[3], w[3], gw[3], t[3], gdn[3], gdd[3];
                    for (int i = 0; i < 3; i++) dd[i] = dn[i] = C(br.i1)[i] - C(br.i2)[i];
                    vect_normalize(dn);
                    cross(rv, dn, w);
                    normalize_bwd(w, grv2, gw, false);
                    cross(dn, gw, t);  // d(rv x dn)/d rv ^T gw
                    for (int i = 0; i < 3; i++) g_rv_t[i] += t[i];
                    cross(gw, rv, gdn);  // d(rv x dn)/d dn ^T gw
                    normalize_bwd(dd, gdn, gdd, false);
                    add(br.i1, gdd, 1.);
                    add(br.i2, gdd, -1.);
                }
                double gu[3];
                normalize_bwd(u, g_rv_t, gu, true);
                add(ia, gu, 1.);
                add(br.i1, gu, -1.);
            } break;
            case BondRec::A2_DIS: {
                double u[3], gu[3];
                for (int i = 0; i < 3; i++) u[i] = C(ia)[i] - C(br.i1)[i];
                normalize_bwd(u, grv, gu, true);
                add(ia, gu, 1.);
                add(br.i1, gu, -1.);
            } break;
            case BondRec::A2_TWO: {
                double er[3], e[3], s[3], v[3], gv[3];
                for (int i = 0; i < 3; i++) { er[i] = C(br.i2)[i] - C(br.i1)[i]; s[i] = C(ia)[i] - C(br.i1)[i]; }
                vect_sub_normalize(e, C(br.i2), C(br.i1));
                double rdot = 0.;
                for (int i = 0; i < 3; i++) rdot += s[i] * e[i];
                for (int i = 0; i < 3; i++) v[i] = C(ia)[i] - ((rdot * e[i]) + C(br.i1)[i]);
                normalize_bwd(v, grv, gv, false);
                const double egv = e[0] * gv[0] + e[1] * gv[1] + e[2] * gv[2];
                double gs[3], ge[3], ger[3];
                for (int i = 0; i < 3; i++) {
                    gs[i] = gv[i] - e[i] * egv;                       // v = s - (s.e) e
                    ge[i] = grv2[i] - (rdot * gv[i] + egv * s[i]);
                }
                normalize_bwd(er, ge, ger, true);
                add(br.i2, ger, 1.);
                add(br.i1, ger, -1.);
                add(ia, gs, 1.);
                add(br.i1, gs, -1.);
            } break;
            case BondRec::A1: {
                if (br.nb == 0) break;
                double mean[3] = {0, 0, 0}, gm[3], gmean[3];
                for (int b = 0; b < br.nb; b++)
                    for (int i = 0; i < 3; i++) mean[i] += (C(ia)[i] - C(br.nbr[b])[i]) / br.nb;
                for (int i = 0; i < 3; i++) gm[i] = -grv[i];
                normalize_bwd(mean, gm, gmean, false);
                add(ia, gmean, 1.);
                for (int b = 0; b < br.nb; b++) add(br.nbr[b], gmean, -1. / br.nb);
            } break;
            default: break;
        }
    }
}

// main.cpp:2684-2736
void Job::build_disorder()
{
    for (int ia = 0; ia < n_atoms; ia++) {
        int hcount = 0;
        for (int b = 0; b < kMaxNBonds && b < nbonds[ia]; b++)
            if (atom_type[bonded[ia][b]] == hydrogen) hcount++;
        const int t = atom_type[ia];
        if ((t == nitrogen && hcount == 2) || (t == nonHB_nitrogen && hcount == 3) ||
            (t == oxygen && hcount == 1) || (t == sulphur && hcount == 1)) {
            disorder[ia] = 1;
            for (int b = 0; b < kMaxNBonds && b < nbonds[ia]; b++) {
                int ba = bonded[ia][b];
                if (atom_type[ba] == hydrogen) disorder[ba] = 1;
            }
        }
    }
}

// xs radii of read_parameter_library.cc:323-339 (an ADVINA-only table in the
// reference); 1.8 for a type missing from it (:352-354).
static double vina_xs_radius(const std::string &t)
{
    static const struct { const char *name; float value; } kXs[] = {
        {"C", 1.9f}, {"A", 1.9f}, {"N", 1.8f}, {"NA", 1.8f}, {"NS", 1.8f}, {"O", 1.7f}, {"OA", 1.7f},
        {"OS", 1.7f}, {"S", 2.0f}, {"SA", 2.0f}, {"P", 2.1f}, {"F", 1.5f}, {"Mg", 1.2f}};
    for (const auto &e : kXs)
        if (t == e.name) return (double)e.value;
    return (double)1.8f;
}

// Vina-potential tables of main.cpp:2081-2126 (compiled out of the reference
// build by use_vina_potential = FALSE, main.cpp:263), restated as written:
// float weights, float table accumulating each term in turn, bin 0 left at
// zero, no smoothing.  The terms act on the surface distance
// d = r - (xs(receptor type) + xs(ligand type)): two Gaussians, d^2 repulsion
// for d < 0, the H-bond step for hbonder pairs (d <= 0.7 adds the weight, and
// -0.7 < d <= 0 subtracts (d/0.7) of it), and the hydrophobic step for pairs
// that are hbonders neither way -- the second test reads gridmap[i].hbonder[ia]
// with the receptor-type index i as a map index (main.cpp:2117), restated with
// 0 where that map does not exist.
// The problem keeps the job's atoms and grid; its maps are the atom maps only
// (the reference skips the e and d maps and desolvation under Vina,
// main.cpp:2968, :3379, :3391) and every pair term is a plain sum.
void Job::build_vina_problem()
{
    if (vina_built) return;
    if (separate_desolvation_maps) fatal("separate_desolvation_maps has no Vina counterpart", AG_ERR_UNSUPPORTED);
    const double wt_gauss1 = (double)-0.035579f, wt_gauss2 = (double)-0.005156f;
    const double wt_repulsion = (double)0.840245f, wt_hydrogen = (double)-0.587439f;
    const double wt_hydrophobic = (double)-0.035069f;
    const int nR = std::max(receptor_types_ct, 1), nAM = std::max(num_atom_maps, 1);
    vina_tab.assign((size_t)nR * nAM * AG_NEINT, 0.0f);
    for (int ia = 0; ia < num_atom_maps; ia++) {
        const MapObj &g = gridmap[ia];
        if (g.is_covalent) continue;
        const double Rij = vina_xs_radius(ligand_types[ia]);
        for (int i = 0; i < receptor_types_ct; i++) {
            const float map_Rij = (float)vina_xs_radius(receptor_types[i]);
            float *t = &vina_tab[((size_t)i * num_atom_maps + ia) * AG_NEINT];
            const int alias = (i < num_maps && ia < AG_MAX_REC_TYPES) ? gridmap[i].hbonder[ia] : 0;
            for (int k = 1; k < AG_NEINT; k++) {
                const double r = angstrom(k);
                const double d = r - (map_Rij + Rij);
                double de = wt_gauss1 * std::exp(-std::pow(d / 0.5, 2)) + wt_gauss2 * std::exp(-std::pow((d - 3.) / 2., 2));
                t[k] = (float)((double)t[k] + de);
                if (d < 0) t[k] = (float)((double)t[k] + wt_repulsion * std::pow(d, 2));
                if (g.hbonder[i] > 0) {
                    if (d <= 0.7) t[k] = (float)((double)t[k] + 1 * wt_hydrogen);
                    if ((-0.7 < d) && (d <= 0.)) t[k] = (float)((double)t[k] - (d / 0.7) * wt_hydrogen);
                }
                if (g.hbonder[i] == 0 && alias == 0) {
                    de = 0.;
                    if (d < 0.5) de = 1 * wt_hydrophobic;
                    else if (d < 1.5) de = (0.5 - d) * wt_hydrophobic;
                    t[k] = (float)((double)t[k] + de);
                }
            }
        }
    }
    vina_is_hb.assign(nAM, 0);
    vina_zero.assign(nAM, 0.0);
    vina_prob = prob;
    vina_prob.n_maps = num_atom_maps;
    vina_prob.elec_map = -1;
    vina_prob.dsolv_map = -1;
    vina_prob.map_is_hbonder = vina_is_hb.data();
    vina_prob.map_solpar_probe = vina_zero.data();
    vina_prob.map_vol_probe = vina_zero.data();
    vina_prob.e_vdw_hb = vina_tab.data();
    vina_prob.separate_desolvation_maps = 0;
    vina_built = true;
}

void Job::make_problem()
{
    m_is_cov.assign(std::max(num_atom_maps, 1), 0);
    m_is_hb.assign(std::max(num_atom_maps, 1), 0);
    m_hbond.assign(std::max(num_atom_maps, 1), 0);
    m_solpar.assign(std::max(num_atom_maps, 1), 0.0);
    m_vol.assign(std::max(num_atom_maps, 1), 0.0);
    for (int i = 0; i < num_atom_maps; i++) {
        m_is_cov[i] = gridmap[i].is_covalent;
        m_is_hb[i] = gridmap[i].is_hbonder;
        m_hbond[i] = gridmap[i].hbond;
        m_solpar[i] = gridmap[i].solpar_probe;
        m_vol[i] = gridmap[i].vol_probe;
    }
    if (r_epsilon_fn.size() != AG_NDIEL) r_epsilon_fn.assign(AG_NDIEL, 0.0);
    ag_problem &p = prob;
    std::memset(&p, 0, sizeof p);
    p.n_atoms = n_atoms;
    p.coord = coord.data();
    p.charge = charge.data();
    p.vol = vol.data();
    p.solpar = solpar.data();
    p.rec_type = atom_type.data();
    p.hbond = hbond.data();
    p.rexp = rexp.data();
    p.rvector = rvector.data();
    p.rvector2 = rvector2.data();
    p.disorder = disorder.data();
    for (int i = 0; i < 3; i++) { p.n1[i] = n1[i]; p.ne[i] = ne[i]; }
    p.spacing = spacing;
    p.n_rec_types = receptor_types_ct;
    p.n_atom_maps = num_atom_maps;
    p.n_maps = num_maps;
    p.elec_map = elecPE;
    p.dsolv_map = dsolvPE;
    p.map_is_covalent = m_is_cov.data();
    p.map_is_hbonder = m_is_hb.data();
    p.map_hbond = m_hbond.data();
    p.map_solpar_probe = m_solpar.data();
    p.map_vol_probe = m_vol.data();
    p.e_vdw_hb = e_vdw_hb.data();
    p.sol_fn = sol_fn.data();
    p.r_epsilon_fn = r_epsilon_fn.data();
    p.dddiel = dddiel ? 1 : 0;
    p.invdielcal = invdielcal;
    p.coeff_estat = ad4.coeff_estat;
    p.solpar_q = solpar_q;
    p.disorder_h = disorder_h ? 1 : 0;
    p.hydrogen_type = hydrogen;
    p.separate_desolvation_maps = separate_desolvation_maps ? 1 : 0;
    for (int i = 0; i < 3; i++) p.cov_pos[i] = covpos[i];
    p.cov_half_width = covhalfwidth;
    p.cov_barrier = covbarrier;
    p.floating_grid = floating_grid ? 1 : 0;
    p.constriction_grid = constriction_grid ? 1 : 0;
    p.constriction_cutoff = constriction_cutoff;
    p.report_collisions = map_receptor_interior ? 0 : 1;
}

// ------------------------------------------------------------- map writer --
// main.cpp:3481-3565.  write_maps formats on the host; write_text takes bodies
// formatted on the device by ag_maps_format (same bytes).
void Job::write_maps(const double *m64, const float *m32)
{
    const size_t P = (size_t)num_grid_points_per_map;
    const size_t n_out = (size_t)num_maps + (floating_grid ? 1 : 0) + (constriction_grid ? 1 : 0);
    auto val = [&](size_t k, size_t a) { return m64 ? m64[k * P + a] : (double)m32[k * P + a]; };
    std::vector<char> text;
    text.reserve(P * n_out * 8 + 64);
    std::vector<size_t> bytes(n_out, 0);
    std::vector<double> emin((size_t)num_maps, kBig), emax((size_t)num_maps, -kBig);
    char tmp[64];
    for (size_t k = 0; k < n_out; k++) {
        const size_t before = text.size();
        const bool energy = k < (size_t)num_maps, count = !energy && !(floating_grid && k == (size_t)num_maps);
        for (size_t a = 0; a < P; a++) {
            const double e = val(k, a);
            int n;
            if (count) {
                n = std::snprintf(tmp, sizeof tmp, "%d\n", (int)e);
            } else if (energy && std::fabs(e) < kPrecision) {
                tmp[0] = '0'; tmp[1] = '\n'; n = 2;
            } else {
                const float v = (float)(std::round((long double)e * 1000.0L) / 1000.0L);  // round3dp, main.cpp:86
                n = std::snprintf(tmp, sizeof tmp, "%.3f\n", (double)v);
            }
            text.insert(text.end(), tmp, tmp + n);
            if (energy) {
                emax[k] = std::max(emax[k], e);
                emin[k] = std::min(emin[k], e);
            }
        }
        bytes[k] = text.size() - before;
    }
    write_text(text.data(), bytes.data(), emin.data(), emax.data());
}

void Job::write_text(const char *text, const size_t *bytes, const double *emin, const double *emax)
{
    const size_t n_out = (size_t)num_maps + (floating_grid ? 1 : 0) + (constriction_grid ? 1 : 0);
    std::vector<std::FILE *> fps;
    for (int j = 0; j < num_maps; j++) fps.push_back(gridmap[j].fp);
    if (floating_grid) fps.push_back(floating_fp);
    if (constriction_grid) fps.push_back(constriction_fp);
    std::vector<size_t> off(n_out + 1, 0);
    for (size_t k = 0; k < n_out; k++) off[k + 1] = off[k] + bytes[k];
    // one file per thread, as the reference's loop over maps is an OpenMP
    // parallel for (main.cpp:3484)
    std::vector<char> failed(n_out, 0);
    const size_t nt = std::min<size_t>(n_out, 16);
    std::vector<std::thread> pool;
    for (size_t t = 0; t < nt; t++)
        pool.emplace_back([&, t] {
            for (size_t k = t; k < n_out; k += nt) {
                if (!fps[k]) continue;
                if (std::fwrite(text + off[k], 1, bytes[k], fps[k]) != bytes[k]) failed[k] = 1;
                if (std::fclose(fps[k]) != 0) failed[k] = 1;
            }
        });
    for (auto &th : pool) th.join();
    for (int j = 0; j < num_maps; j++) {
        gridmap[j].fp = nullptr;
        if (emin) gridmap[j].emin = std::min(gridmap[j].emin, emin[j]);
        if (emax) gridmap[j].emax = std::max(gridmap[j].emax, emax[j]);
    }
    if (floating_grid) floating_fp = nullptr;
    if (constriction_grid) constriction_fp = nullptr;
    bool problem = false;
    for (char f : failed) problem = problem || f;
    if (problem) fatal("Problems writing grid maps - there may not be enough disk space.", AG_ERR_IO);
    log("\nGrid\tAtom\tMinimum   \tMaximum\nMap \tType\tEnergy    \tEnergy \n\t\t(kcal/mol)\t(kcal/mol)\n"
        "____\t____\t_____________\t_____________\n");
    for (int i = 0; i < num_atom_maps; i++)
        log(fmt(" %d\t %s\t  %6.2lf\t%9.2le\n", i + 1, gridmap[i].type.c_str(), gridmap[i].emin, gridmap[i].emax));
    if (elecPE >= 0)
        log(fmt(" %d\t %c\t  %6.2lf\t%9.2le\tElectrostatic Potential\n", elecPE + 1, 'e', gridmap[elecPE].emin,
                gridmap[elecPE].emax));
    if (dsolvPE >= 0)
        log(fmt(" %d\t %c\t  %6.2lf\t%9.2le\tDesolvation Potential\n", dsolvPE + 1, 'd', gridmap[dsolvPE].emin,
                gridmap[dsolvPE].emax));
    log(fmt("\n\n * Note:  Every pairwise-atomic interaction was clamped at %.2f\n\n", kEintClamp));
    const double secs = (double)(clock() - t_start) / CLOCKS_PER_SEC;
    log(fmt("\n%s: Successful Completion.\n", kProgram));
    log(fmt("Real= %.2fs\n", secs));
    finished = true;
}

}  // namespace agb

// ================================================================ C ABI ====
using agb::Fatal;
using agb::Job;

struct ag_job {
    Job job;
};

extern "C" {

ag_status ag_job_load(const char *gpf_path, const char *glg_path, ag_job **out)
{
    if (!gpf_path || !out) { agb::set_last_error("ag_job_load: null argument"); return AG_ERR_INVALID; }
    *out = nullptr;
    ag_job *j = new ag_job();
    j->job.t_start = clock();
    if (glg_path) {
        j->job.glg = std::fopen(glg_path, "w");
        if (!j->job.glg) {
            agb::set_last_error(std::string("can't create the log file ") + glg_path);
            delete j;
            return AG_ERR_IO;
        }
        j->job.glg_owned = true;
    } else {
        j->job.glg = stdout;
    }
    j->job.log("\n       AutoGrid-B200 (AutoGrid 4 map engine for NVIDIA B200)\n\n");
    try {
        j->job.load(gpf_path);
    } catch (const Fatal &f) {
        ag_job_fail(j, f.what());
        agb::set_last_error(f.what());
        ag_status s = f.status;
        delete j;
        return s;
    } catch (const std::exception &e) {
        ag_job_fail(j, e.what());
        agb::set_last_error(e.what());
        delete j;
        return AG_ERR_INVALID;
    }
    *out = j;
    return AG_OK;
}

const ag_problem *ag_job_problem(const ag_job *job) { return job ? &job->job.prob : nullptr; }

static ag_status write_common(ag_job *job, const double *m64, const float *m32)
{
    if (!job || (!m64 && !m32)) { agb::set_last_error("ag_job_write_maps: null argument"); return AG_ERR_INVALID; }
    try {
        job->job.write_maps(m64, m32);
    } catch (const Fatal &f) {
        ag_job_fail(job, f.what());
        agb::set_last_error(f.what());
        return f.status;
    }
    return AG_OK;
}

ag_status ag_job_write_maps_f32(ag_job *job, const float *maps) { return write_common(job, nullptr, maps); }
ag_status ag_job_write_maps_f64(ag_job *job, const double *maps) { return write_common(job, maps, nullptr); }

ag_status ag_job_write_text(ag_job *job, const char *text, const size_t *map_bytes, const double *emin,
                            const double *emax)
{
    if (!job || !text || !map_bytes) { agb::set_last_error("ag_job_write_text: null argument"); return AG_ERR_INVALID; }
    try {
        job->job.write_text(text, map_bytes, emin, emax);
    } catch (const Fatal &f) {
        ag_job_fail(job, f.what());
        agb::set_last_error(f.what());
        return f.status;
    }
    return AG_OK;
}

void ag_job_fail(ag_job *job, const char *message)
{
    if (!job) return;
    job->job.log(agb::fmt("\n%s: ERROR:  %s\n\n", "autogrid4_b200", message ? message : ""));
    job->job.log(agb::fmt("\n%s: Unsuccessful Completion.\n", "autogrid4_b200"));
}

void ag_job_free(ag_job *job) { delete job; }

ag_status ag_job_vina_problem(ag_job *job, const ag_problem **out)
{
    if (!job || !out) { agb::set_last_error("ag_job_vina_problem: null argument"); return AG_ERR_INVALID; }
    *out = nullptr;
    try {
        job->job.build_vina_problem();
    } catch (const Fatal &f) {
        agb::set_last_error(f.what());
        return f.status;
    }
    *out = &job->job.vina_prob;
    return AG_OK;
}

ag_status ag_job_bond_vectors(const ag_job *job, const double *coord, double *rvector, double *rvector2)
{
    if (!job || !rvector || !rvector2) { agb::set_last_error("ag_job_bond_vectors: null argument"); return AG_ERR_INVALID; }
    job->job.eval_bond_vectors(coord ? coord : job->job.coord.data(), rvector, rvector2);
    return AG_OK;
}

ag_status ag_job_bond_vectors_backward(const ag_job *job, const double *coord, const double *g_rvector,
                                       const double *g_rvector2, double *g_coord)
{
    if (!job || !g_rvector || !g_rvector2 || !g_coord) {
        agb::set_last_error("ag_job_bond_vectors_backward: null argument");
        return AG_ERR_INVALID;
    }
    job->job.bond_vectors_backward(coord ? coord : job->job.coord.data(), g_rvector, g_rvector2, g_coord);
    return AG_OK;
}

ag_status ag_job_table_params(const ag_job *job, ag_table_params *out)
{
    if (!job || !out) { agb::set_last_error("ag_job_table_params: null argument"); return AG_ERR_INVALID; }
    Job &j = const_cast<ag_job *>(job)->job;
    const int nT = j.receptor_types_ct, nAM = j.num_atom_maps;
    const size_t n = (size_t)std::max(0, nT) * std::max(0, nAM);
    j.tp_cA.assign(n, 0.); j.tp_cB.assign(n, 0.); j.tp_R.assign(n, 0.); j.tp_eps.assign(n, 0.);
    j.tp_xA.assign(n, 0); j.tp_xB.assign(n, 0); j.tp_cov.assign((size_t)std::max(nAM, 0), 0);
    for (int m = 0; m < nAM; m++) {
        const auto &g = j.gridmap[m];
        j.tp_cov[m] = g.is_covalent;
        for (int t = 0; t < nT; t++) {
            const size_t k = (size_t)m * nT + t;
            j.tp_cA[k] = g.cA[t]; j.tp_cB[k] = g.cB[t]; j.tp_R[k] = g.nbp_r[t]; j.tp_eps[k] = g.nbp_eps[t];
            j.tp_xA[k] = g.xA[t]; j.tp_xB[k] = g.xB[t];
        }
    }
    out->n_rec_types = nT;
    out->n_atom_maps = nAM;
    out->cA = j.tp_cA.data(); out->cB = j.tp_cB.data(); out->Rij = j.tp_R.data(); out->epsij = j.tp_eps.data();
    out->xA = j.tp_xA.data(); out->xB = j.tp_xB.data(); out->map_is_covalent = j.tp_cov.data();
    out->r_smooth = j.r_smooth;
    out->coeff_desolv = j.ad4.coeff_desolv;
    out->dddiel = j.dddiel ? 1 : 0;
    return AG_OK;
}

ag_status ag_job_bond_topology(const ag_job *job, int32_t *topo)
{
    if (!job || !topo) { agb::set_last_error("ag_job_bond_topology: null argument"); return AG_ERR_INVALID; }
    static_assert(agb::BondRec::D1 == AG_BOND_D1 && agb::BondRec::A2_ONE == AG_BOND_A2_ONE &&
                      agb::BondRec::A2_DIS == AG_BOND_A2_DIS && agb::BondRec::A2_TWO == AG_BOND_A2_TWO &&
                      agb::BondRec::A1 == AG_BOND_A1,
                  "bond kinds");
    const auto &br = job->job.bondrec;
    for (size_t a = 0; a < br.size(); a++) {
        int32_t *t = topo + 7 * a;
        t[0] = br[a].kind;
        t[1] = br[a].i1;
        t[2] = br[a].i2;
        t[3] = br[a].nb;
        for (int b = 0; b < 3; b++) t[4 + b] = br[a].nbr[b];
    }
    return AG_OK;
}

const char *ag_last_error(void) { return agb::last_error(); }
int32_t ag_abi_version(void) { return AG_ABI_VERSION; }

}  // extern "C"
