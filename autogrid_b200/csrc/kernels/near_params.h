// Parameters shared by the host orchestration and the near-field kernel.
#pragma once
#include <cstdint>

namespace agb {

constexpr int NG_MAX = 16;                 // ligand maps per near-kernel launch
constexpr int NG_MM = 4;                   // of which at most this many keep hbond min/max (placed first)
constexpr int NT_SMALL = 1040;             // table bins a near pair can reach (r <= 8 A + guard)
constexpr int NB_CHUNK_MAX = 384;          // near candidates staged in shared memory at once
constexpr int NB_WARPS_MAX = 8;            // warps of a near-kernel CTA (256 threads)
constexpr int NB_THREADS_MAX = NB_WARPS_MAX * 32;
constexpr int NB_SEGS_MAX = 64;            // cell-row segments laid out at once
constexpr double AGB_NEAR_RADIUS = 8.05;   // A; > 8 A cutoff + FP32 distance error
constexpr double AGB_CELL = 4.0;           // A; cell-list edge

// What one (ligand map, receptor-atom hbond class) pair contributes, after
// main.cpp:3286-3379.  Desolvation is handled separately (factored).
enum : uint8_t {
    ACT_SKIP = 0,  // covalent map, or the desolvation partner of a separate_desolvation_maps pair
    ACT_PLAIN,     // E += T
    ACT_SUMA,      // probe acceptor vs receptor donor: E += T*Hramp*(racc+(1-racc)rsph)
    ACT_MMA,       // A1/AD probe vs donor: hbondmin/max of T*(racc+(1-racc)rsph)
    ACT_MMD        // donor probe vs acceptor: hbondmin/max of T*(rdon+(1-rdon)rsph)
};

struct NearGroup {
    int ng;                    // ligand maps handled by this launch, in kernel order
    int write_special;         // this launch also writes the d and e maps
    int has_hrow;              // some action reads the hydrogen row (disorder_h)
    int col0;                  // first column of this launch's maps in the [type][bin][col] table
    unsigned long long actw[8];  // per receptor hbond class: 3-bit action of kernel map m at bits 3m..3m+2
    unsigned plain_hb;         // bit hb: every map of this launch is ACT_PLAIN or ACT_SKIP for class hb
                               // (the table columns of ACT_SKIP maps are zero, so all T can be added)
    unsigned plain4;           // bit 4*hb + r: kernel maps 4r..4r+3 (one 16-byte table row) are all
                               // ACT_PLAIN or ACT_SKIP for class hb, so the row adds as a whole
    int out_map[NG_MAX];       // output map index of kernel map m
    uint8_t cov[NG_MAX];
    double sp[NG_MAX], vp[NG_MAX];  // desolvation factors applied to this map's output
};

}  // namespace agb
