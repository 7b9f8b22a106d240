// Host check of the differentiable mode's per-pair arithmetic
// (autogrid_b200/csrc/kernels/diff_pair.cuh, the code the kernels run),
// instantiated in FP64 on the CPU: the adjoint (pair_bwd + angular_bwd +
// geom_bwd, plus the closest-hydrogen ramp term) against central differences
// of the forward (pair_fwd + the H-bond min/max finaliser) for random atoms of
// every hbond class, random bond vectors, random points within 8 A and smooth
// random tables.  Prints the worst relative error and exits 1 above 1e-5
// (central differences with h = 1e-6 on losses of order 1e6 carry ~1e-6 of
// rounding).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "kernels/diff_pair.cuh"

using namespace agb;
using namespace agb::dfm;

namespace {

constexpr int NT = 6, NAM = 6, NA = 48, NP = 40;

struct Case {
    DiffArgs a{};
    std::vector<R2<double>> vdw, sol;
    std::vector<Atom<double>> atoms;
    std::vector<double> px, py, pz, w;  // points, loss weights [NP][n_slots]
    std::vector<int> ch;
};

// slot s of type t: rows [t][bin][stride]
void make_table(std::vector<R2<double>> &tab, int t, int s, int stride, double A, double B, double clamp)
{
    std::vector<double> v(AG_NEINT);
    for (int b = 0; b < AG_NEINT; b++) {
        const double r = std::max(b, 1) / 128.0;
        v[b] = std::min(A / std::pow(r, 12) - B / std::pow(r, 6), clamp);
    }
    v[AG_NEINT - 1] = 0;
    for (int b = 0; b < AG_NEINT; b++)
        tab[((size_t)t * AG_NEINT + b) * stride + s] = R2<double>{v[b], b < AG_NEINT - 1 ? v[b + 1] - v[b] : 0.0};
}

double loss(const Case &c, const std::vector<Atom<double>> &atoms)
{
    const DiffArgs &a = c.a;
    double L = 0;
    for (int p = 0; p < NP; p++) {
        double E[DF_MAXS] = {}, hmin[DF_MAXMM], hmax[DF_MAXMM];
        int amin[DF_MAXMM], amax[DF_MAXMM];
        for (int s = 0; s < DF_MAXMM; s++) { hmin[s] = 999999.; hmax[s] = -999999.; amin[s] = amax[s] = -1; }
        const int ch = c.ch[p];
        const double *rvh = atoms[ch].rv;
        for (const auto &at : atoms) {
            Geom<double> g;
            if (!geom(c.sol.data(), at, c.px[p], c.py[p], c.pz[p], g)) continue;
            Ang<double> an;
            angular((at.meta >> DM_HB_SHIFT) & 7, (at.meta >> DM_REXP_SHIFT) & 7, (at.meta & DM_DIS) != 0,
                    at.idx != ch, g.dn, at.rv, at.rv2, rvh, an);
            pair_fwd(a, c.vdw.data(), g, at, an, E, hmin, hmax, amin, amax);
        }
        for (int s = 0; s < a.n_slots; s++) {
            double v = E[s];
            if (s < a.n_mm && amin[s] >= 0) v += hmin[s] + std::max(hmax[s], 0.0);
            L += c.w[p * a.n_slots + s] * v;
        }
    }
    return L;
}

// analytic gradient: [atom][coord 3, q, rv 3, rv2 3]
void grad(const Case &c, std::vector<double> &G)
{
    const DiffArgs &a = c.a;
    G.assign((size_t)NA * 10, 0.0);
    for (int p = 0; p < NP; p++) {
        double E[DF_MAXS] = {}, hmin[DF_MAXMM], hmax[DF_MAXMM];
        int amin[DF_MAXMM], amax[DF_MAXMM];
        for (int s = 0; s < DF_MAXMM; s++) { hmin[s] = 999999.; hmax[s] = -999999.; amin[s] = amax[s] = -1; }
        const int ch = c.ch[p];
        const double *rvh = c.atoms[ch].rv;
        for (const auto &at : c.atoms) {
            Geom<double> g;
            if (!geom(c.sol.data(), at, c.px[p], c.py[p], c.pz[p], g)) continue;
            Ang<double> an;
            angular((at.meta >> DM_HB_SHIFT) & 7, (at.meta >> DM_REXP_SHIFT) & 7, (at.meta & DM_DIS) != 0,
                    at.idx != ch, g.dn, at.rv, at.rv2, rvh, an);
            pair_fwd(a, c.vdw.data(), g, at, an, E, hmin, hmax, amin, amax);
        }
        for (int s = 0; s < DF_MAXMM; s++)
            if (!(hmax[s] > 0)) amax[s] = -1;
        double gs[DF_MAXS] = {};
        for (int s = 0; s < a.n_slots; s++) gs[s] = c.w[p * a.n_slots + s];
        double g_rvh[3] = {0, 0, 0};
        for (const auto &at : c.atoms) {
            Geom<double> g;
            if (!geom(c.sol.data(), at, c.px[p], c.py[p], c.pz[p], g)) continue;
            const int hb = (at.meta >> DM_HB_SHIFT) & 7;
            const bool dis = (at.meta & DM_DIS) != 0;
            Ang<double> an;
            angular(hb, (at.meta >> DM_REXP_SHIFT) & 7, dis, at.idx != ch, g.dn, at.rv, at.rv2, rvh, an);
            double Gx = 0, Gracc = 0, Grdon = 0, GH = 0, Gq = 0;
            pair_bwd(a, c.vdw.data(), g, at, an, gs, amin, amax, Gx, Gracc, Grdon, GH, Gq);
            double g_dn[3] = {0, 0, 0}, g_rv[3] = {0, 0, 0}, g_rv2[3] = {0, 0, 0}, g_d[3];
            angular_bwd(hb, dis, an, Gracc, Grdon, GH, g.dn, at.rv, at.rv2, rvh, g_dn, g_rv, g_rv2, g_rvh);
            geom_bwd(g, Gx, g_dn, g_d);
            double *o = &G[(size_t)at.idx * 10];
            for (int i = 0; i < 3; i++) { o[i] += g_d[i]; o[4 + i] += g_rv[i]; o[7 + i] += g_rv2[i]; }
            o[3] += Gq;
        }
        for (int i = 0; i < 3; i++) G[(size_t)ch * 10 + 4 + i] += g_rvh[i];
    }
}

double &param(std::vector<Atom<double>> &atoms, int a, int k)
{
    Atom<double> &t = atoms[a];
    switch (k) {
        case 0: return t.x;
        case 1: return t.y;
        case 2: return t.z;
        case 3: return t.q;
        default: return k < 7 ? t.rv[k - 4] : t.rv2[k - 7];
    }
}

}  // namespace

int main(int argc, char **argv)
{
    const unsigned seed = argc > 1 ? (unsigned)std::atoi(argv[1]) : 1u;
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> U(-1, 1);
    std::normal_distribution<double> Nd(0, 1);
    Case c;
    DiffArgs &a = c.a;
    a.n_atoms = NA;
    a.n_atom_maps = NAM;
    a.n_rec_types = NT;
    a.solpar_q = 0.01097;
    a.hydrogen_type = 2;  // < NT
    // slots: 2 min/max maps (A1 probe "NA", donor probe "HD"), 3 plain/acceptor maps, 1 d map
    const int map_hbond[NAM] = {4, 2, 0, 5, 3, 0};
    a.n_slots = NAM + 1;
    a.n_mm = 2;
    for (int s = 0; s < NAM; s++) {
        a.slot_map[s] = s;
        a.slot_kind[s] = DK_ATOM;
        a.slot_tab[s] = s;
        a.slot_desolv[s] = 1;
        a.slot_sp[s] = 0.01 + 0.002 * s;
        a.slot_vp[s] = 10.0 + s;
        const int mh = map_hbond[s];
        for (int dis = 0; dis < 2; dis++)
            for (int hb = 0; hb < 8; hb++) {
                uint8_t act = DA_PLAIN;
                const bool donor = hb == 1 || hb == 2 || hb == 6;
                if (mh != 0) {
                    if ((mh == 3 || mh == 5 || mh == 6) && donor) act = dis ? DA_SUMA_DIS : DA_SUMA;
                    else if ((mh == 4 || mh == 6) && donor) act = DA_MMA;
                    else if ((mh == 1 || mh == 2 || mh == 6) && (hb > 2 || hb == 6)) act = dis ? DA_SUMD_DIS : DA_MMD;
                }
                a.act[s][hb + 8 * dis] = act;
            }
    }
    a.slot_map[NAM] = NAM;
    a.slot_kind[NAM] = DK_D;
    a.slot_tab[NAM] = -1;
    a.tab_stride = 8;
    c.vdw.assign((size_t)NT * AG_NEINT * a.tab_stride, R2<double>{0, 0});
    for (int t = 0; t < NT; t++)
        for (int m = 0; m < NAM; m++)
            make_table(c.vdw, t, m, a.tab_stride, 2000.0 * (1 + 0.3 * t) * (1 + 0.1 * m), 40.0 * (1 + 0.2 * m),
                       100000.0);
    c.sol.resize(AG_NEINT);
    std::vector<double> sv(AG_NEINT + 1);
    for (int b = 0; b <= AG_NEINT; b++) { const double r = b / 128.0; sv[b] = 0.1711 * std::exp(-r * r / 25.92); }
    for (int b = 0; b < AG_NEINT; b++) c.sol[b] = R2<double>{sv[b], sv[b + 1] - sv[b]};

    // atoms: every class; unit bond vectors; D1 rexp 1/2/4; a few disordered
    const int classes[] = {0, 1, 2, 2, 2, 4, 5, 5, 5, 6};
    for (int i = 0; i < NA; i++) {
        Atom<double> t{};
        t.x = 4 * U(rng); t.y = 4 * U(rng); t.z = 4 * U(rng);
        t.q = 0.3 * Nd(rng); t.vol = 10 + 10 * std::abs(U(rng)); t.solpar = -0.001 + 0.002 * U(rng);
        const int hb = classes[i % 10];
        const bool dis = (hb == 5 && i % 3 == 0) || (hb == 2 && i % 7 == 0);
        const int rexp = (i % 3 == 0) ? 1 : (i % 3 == 1 ? 2 : 4);
        const int type = i % NT;
        double v[3] = {Nd(rng), Nd(rng), Nd(rng)}, n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        for (int k = 0; k < 3; k++) t.rv[k] = (hb == 2 || hb == 4 || hb == 5) ? v[k] / n : 0.0;
        double u[3] = {Nd(rng), Nd(rng), Nd(rng)};
        n = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        for (int k = 0; k < 3; k++) t.rv2[k] = (hb == 5 && !dis && i % 4 != 1) ? u[k] / n : 0.0;
        t.meta = type | (hb << DM_HB_SHIFT) | (rexp << DM_REXP_SHIFT) | (dis ? DM_DIS : 0);
        t.idx = i;
        c.atoms.push_back(t);
    }
    std::vector<int> d1;
    for (int i = 0; i < NA; i++)
        if (((c.atoms[i].meta >> DM_HB_SHIFT) & 7) == 2) d1.push_back(i);
    for (int p = 0; p < NP; p++) {
        c.px.push_back(3 * U(rng)); c.py.push_back(3 * U(rng)); c.pz.push_back(3 * U(rng));
        c.ch.push_back(d1[rng() % d1.size()]);
        for (int s = 0; s < a.n_slots; s++) c.w.push_back(Nd(rng));
    }

    std::vector<double> G;
    grad(c, G);
    const double h = 1e-6;
    double worst = 0, gmax = 0;
    for (double v : G) gmax = std::max(gmax, std::abs(v));
    int bad_a = -1, bad_k = -1;
    for (int i = 0; i < NA; i++)
        for (int k = 0; k < 10; k++) {
            // a zero rvector2 (no second neighbour) is a constant of the model,
            // and sin(2|ti|) has a kink there
            const Atom<double> &t = c.atoms[i];
            if (k >= 7 && t.rv2[0] == 0 && t.rv2[1] == 0 && t.rv2[2] == 0) continue;
            std::vector<Atom<double>> ap = c.atoms, am = c.atoms;
            param(ap, i, k) += h;
            param(am, i, k) -= h;
            const double fd = (loss(c, ap) - loss(c, am)) / (2 * h);
            const double an = G[(size_t)i * 10 + k];
            const double err = std::abs(fd - an) / std::max(std::abs(fd), 1e-3 * gmax);
            if (err > worst) { worst = err; bad_a = i; bad_k = k; }
        }
    std::printf("seed %u: max |grad| %.4g, worst relative error %.3g (atom %d, parameter %d)\n", seed, gmax, worst,
                bad_a, bad_k);
    return worst <= 1e-5 ? 0 : 1;
}
