// Parameter library: atom_par records and FE_coeff_* weights.
// Semantics follow ad4_shared/read_parameter_library.cc:50-198 (file) and
// :202-398 (built-in defaults), ad4_shared/parse_param_line.cc:42-112 (keyword
// recognition) and atom_parameter_manager.cpp:37-55 (two-character dictionary).
#include <cctype>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <strings.h>

#include "frontend.hpp"

namespace agb {

namespace {

// The AutoDock 4.1 "bound" force field, the reference's compiled-in default
// (its default_parameters.h is generated from ad4_shared/AD4.1_bound.dat).
// These are force-field constants and must be numerically identical.
// Fields: type Rii epsii vol solpar Rij_hb epsij_hb hbond rec_index map_index bond_index
const char *const kAD41Bound[] = {
    "FE_coeff_vdW    0.1662",
    "FE_coeff_hbond  0.1209",
    "FE_coeff_estat  0.1406",
    "FE_coeff_desolv 0.1322",
    "FE_coeff_tors   0.2983",
    "atom_par H      2.00  0.020   0.0000   0.00051  0.0  0.0  0  -1  -1  3",
    "atom_par HD     2.00  0.020   0.0000   0.00051  0.0  0.0  2  -1  -1  3",
    "atom_par HS     2.00  0.020   0.0000   0.00051  0.0  0.0  1  -1  -1  3",
    "atom_par C      4.00  0.150  33.5103  -0.00143  0.0  0.0  0  -1  -1  0",
    "atom_par A      4.00  0.150  33.5103  -0.00052  0.0  0.0  0  -1  -1  0",
    "atom_par N      3.50  0.160  22.4493  -0.00162  0.0  0.0  0  -1  -1  1",
    "atom_par NA     3.50  0.160  22.4493  -0.00162  1.9  5.0  4  -1  -1  1",
    "atom_par NS     3.50  0.160  22.4493  -0.00162  1.9  5.0  3  -1  -1  1",
    "atom_par OA     3.20  0.200  17.1573  -0.00251  1.9  5.0  5  -1  -1  2",
    "atom_par OS     3.20  0.200  17.1573  -0.00251  1.9  5.0  3  -1  -1  2",
    "atom_par F      3.09  0.080  15.4480  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par Mg     1.30  0.875   1.5600  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par MG     1.30  0.875   1.5600  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par P      4.20  0.200  38.7924  -0.00110  0.0  0.0  0  -1  -1  5",
    "atom_par SA     4.00  0.200  33.5103  -0.00214  2.5  1.0  5  -1  -1  6",
    "atom_par S      4.00  0.200  33.5103  -0.00214  0.0  0.0  0  -1  -1  6",
    "atom_par Cl     4.09  0.276  35.8235  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par CL     4.09  0.276  35.8235  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par Ca     1.98  0.550   2.7700  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par CA     1.98  0.550   2.7700  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par Mn     1.30  0.875   2.1400  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par MN     1.30  0.875   2.1400  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par Fe     1.30  0.010   1.8400  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par FE     1.30  0.010   1.8400  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par Zn     1.48  0.550   1.7000  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par ZN     1.48  0.550   1.7000  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par Br     4.33  0.389  42.5661  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par BR     4.33  0.389  42.5661  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par I      4.72  0.550  55.0585  -0.00110  0.0  0.0  0  -1  -1  4",
    "atom_par Z      4.00  0.150  33.5103  -0.00143  0.0  0.0  0  -1  -1  0",
    "atom_par G      4.00  0.150  33.5103  -0.00143  0.0  0.0  0  -1  -1  0",
    "atom_par GA     4.00  0.150  33.5103  -0.00052  0.0  0.0  0  -1  -1  0",
    "atom_par J      4.00  0.150  33.5103  -0.00143  0.0  0.0  0  -1  -1  0",
    "atom_par Q      4.00  0.150  33.5103  -0.00143  0.0  0.0  0  -1  -1  0",
    "atom_par Si     4.10  0.200  35.8235  -0.00143  0.0  0.0  0  -1  -1  6",
    "atom_par B      3.84  0.155  29.6478  -0.00152  0.0  0.0  0  -1  -1  0",
};

enum ParTok { P_NONE = -1, P_NULL, P_COMMENT, P_VDW, P_HBOND, P_ESTAT, P_DESOLV, P_TORS, P_UNBOUND, P_ATOM };

// First word, lower-cased; a keyword matches when the word is a
// case-insensitive prefix of it (parse_param_line.cc:96-104 compares only
// strlen(word) characters).
ParTok classify(const char *line)
{
    char w[256];
    int j = 0;
    while (line[j] && line[j] != ' ' && line[j] != '\t' && line[j] != '\n' && j < 255) {
        w[j] = (char)std::tolower((unsigned char)line[j]);
        j++;
    }
    w[j] = 0;
    if (w[0] == 0 || w[0] == '\n' || w[0] == '\r') return P_NULL;
    if (w[0] == '#') return P_COMMENT;
    static const struct { const char *lex; ParTok t; } tab[] = {
        {"FE_coeff_vdW", P_VDW},     {"FE_coeff_hbond", P_HBOND}, {"FE_coeff_estat", P_ESTAT},
        {"FE_coeff_desolv", P_DESOLV}, {"FE_coeff_tors", P_TORS}, {"FE_unbound_model", P_UNBOUND},
        {"atom_par", P_ATOM}};
    for (auto &e : tab)
        if (strncasecmp(e.lex, w, (size_t)j) == 0) return e.t;
    return P_NONE;
}

}  // namespace

uint32_t ParamLibrary::key(const std::string &t)
{
    if (t.empty()) return 0;
    if (t.size() == 1) return (uint32_t)(unsigned char)t[0];
    return (uint32_t)(unsigned char)t[0] + 256u * (uint32_t)(unsigned char)t[1];
}

ParamEntry *ParamLibrary::find(const std::string &t)
{
    auto it = dict_.find(key(t));
    return it == dict_.end() ? nullptr : &it->second;
}

void ParamLibrary::enter(const ParamEntry &e) { dict_[key(e.type)] = e; }

void ParamLibrary::load_lines(const std::vector<std::string> &lines, FEModel &m)
{
    for (const std::string &s : lines) {
        const char *line = s.c_str();
        ParTok t = classify(line);
        double *coef = nullptr;
        const char *what = nullptr;
        switch (t) {
            case P_VDW: coef = &m.coeff_vdW; what = "van der Waals term"; break;
            case P_HBOND: coef = &m.coeff_hbond; what = "H-bonding term"; break;
            case P_ESTAT: coef = &m.coeff_estat; what = "electrostatic term"; break;
            case P_DESOLV: coef = &m.coeff_desolv; what = "desolvation term"; break;
            case P_TORS: coef = &m.coeff_tors; what = "torsional term"; break;
            case P_UNBOUND:
                throw Fatal(AG_ERR_FATAL_INPUT,
                            "the unbound model cannot be specified in the parameter library file.");
            case P_ATOM: {
                char type[64];
                int rec = last_.rec_index, map = last_.map_index, bidx = last_.bond_index;
                int hb = last_hbond_int_;
                ParamEntry e = last_;
                int n = std::sscanf(line, "%*s %63s %lf %lf %lf %lf %lf %lf %d %d %d %d", type, &e.Rij,
                                    &e.epsij_unweighted, &e.vol, &e.solpar, &e.Rij_hb,
                                    &e.epsij_hb_unweighted, &hb, &rec, &map, &bidx);
                if (n < 2) continue;  // line without enough information is skipped
                e.type = type;
                e.rec_index = rec;
                e.map_index = map;
                e.bond_index = bidx;
                e.hbond = (hb >= 0 && hb <= 5) ? hb : 0;  // read_parameter_library.cc:141-155
                e.epsij = e.epsij_unweighted * m.coeff_vdW;
                e.epsij_hb = e.epsij_hb_unweighted * m.coeff_hbond;
                last_ = e;
                last_hbond_int_ = hb;
                enter(e);
            } break;
            default: break;
        }
        if (coef) {
            if (std::sscanf(line, "%*s %lf", coef) < 1)
                throw Fatal(AG_ERR_FATAL_INPUT, std::string("Must supply a ") + what +
                                                    " coefficient as a floating point number.");
        }
    }
}

void ParamLibrary::load_defaults(FEModel &m)
{
    std::vector<std::string> v(std::begin(kAD41Bound), std::end(kAD41Bound));
    load_lines(v, m);
}

void ParamLibrary::load_file(const std::string &path, FEModel &m)
{
    std::FILE *f = std::fopen(path.c_str(), "r");
    if (!f) throw Fatal(AG_ERR_IO, "Sorry, I can't find or open " + path);
    std::vector<std::string> lines;
    char buf[1024];
    while (std::fgets(buf, sizeof buf, f)) lines.emplace_back(buf);
    std::fclose(f);
    load_lines(lines, m);
}

}  // namespace agb
