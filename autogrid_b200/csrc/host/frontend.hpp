// Internal declarations of the host front end (GPF, parameter library,
// receptor, tables, bond vectors, writers).  Not part of the C ABI.
#pragma once
#include <cstdint>
#include <cstdio>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "autogrid_b200.h"

namespace agb {

// Raised for every condition the reference reports through
// print_error(FATAL_ERROR) (main.cpp:133-177); the C ABI turns it into a
// status code and writes "Unsuccessful Completion" to the GLG.
struct Fatal : std::runtime_error {
    ag_status status;
    Fatal(ag_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};

// Free-energy model coefficients (ad4_shared/structs.h Linear_FE_Model).
struct FEModel {
    double coeff_vdW = 0, coeff_hbond = 0, coeff_estat = 0, coeff_desolv = 0, coeff_tors = 0;
};

// One atom_par record (ad4_shared/structs.h ParameterEntry); rec_index and
// map_index are mutated by the GPF keywords exactly as the reference does.
struct ParamEntry {
    std::string type;
    double Rij = 0, epsij_unweighted = 0, vol = 0, solpar = 0, Rij_hb = 0, epsij_hb_unweighted = 0;
    double epsij = 0, epsij_hb = 0;
    int hbond = 0, rec_index = -1, map_index = -1, bond_index = 0;
};

// The atom-type dictionary.  Keys hash the first two characters only, like
// atom_parameter_manager.cpp:37-43, so "OA" and "OAx" name the same entry.
class ParamLibrary {
  public:
    static uint32_t key(const std::string &t);
    ParamEntry *find(const std::string &t);
    void enter(const ParamEntry &e);
    // setup_parameter_library(): AD4.1 "bound" defaults
    // (ad4_shared/read_parameter_library.cc:202-398, data of AD4.1_bound.dat).
    void load_defaults(FEModel &m);
    // read_parameter_library(): a parameter file (read_parameter_library.cc:50-198).
    void load_file(const std::string &path, FEModel &m);
    void load_lines(const std::vector<std::string> &lines, FEModel &m);

  private:
    std::map<uint32_t, ParamEntry> dict_;
    ParamEntry last_;      // sscanf leaves unparsed fields as they were
    int last_hbond_int_ = 0;
};

}  // namespace agb
