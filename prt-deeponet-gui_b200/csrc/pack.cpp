// pack.cpp -- the placement loop of the synthetic ball packs (host code).
//
// prtlb_gpu.geometry.random_pack draws uniform numbers with numpy and hands
// them over in chunks; this loop places the balls exactly as the NumPy
// version of the same loop does (same accept / reject decisions, same voxels
// stamped), only without the per-try interpreter cost: a candidate is
// tested against the balls of the neighbouring cells of a periodic cell list
// instead of every ball.  Built with -ffp-contract=off so every distance is
// the same IEEE operation sequence as NumPy's.
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "../../include/prtlb.h"

namespace {

struct Pack {
    int nd;
    int shape[3];
    double L[3];
    int ncell[3];
    double csize[3];
    std::unordered_map<long long, std::vector<int>> cells;

    long long key(const int* k) const {
        long long v = 0;
        for (int a = 0; a < nd; ++a) v = v * 1000003LL + k[a];
        return v;
    }
    void cell_of(const double* c, int* k) const {
        for (int a = 0; a < nd; ++a) {
            long long v = (long long)std::floor(c[a] / csize[a]);
            long long m = ncell[a];
            k[a] = (int)(((v % m) + m) % m);
        }
    }
};

// ((d0^2 + d1^2) + d2^2) with periodic minimum image, as NumPy forms
// np.sqrt((np.minimum(|cs - c|, L - |cs - c|) ** 2).sum(1)).
double dist(const Pack& P, const double* a, const double* c) {
    double s = 0.0;
    for (int i = 0; i < P.nd; ++i) {
        double d = std::fabs(a[i] - c[i]);
        const double w = P.L[i] - d;
        d = (w < d) ? w : d;
        const double q = d * d;
        s = (i == 0) ? q : s + q;
    }
    return std::sqrt(s);
}

long long stamp(const Pack& P, uint8_t* solid, const double* c, double r) {
    const int rr = (int)std::ceil(r);
    int base[3] = {0, 0, 0};
    for (int a = 0; a < P.nd; ++a) base[a] = (int)std::floor(c[a]);
    long long added = 0;
    const int span = 2 * rr + 1;
    const int n2 = P.nd == 3 ? span : 1;
    for (int i = 0; i < span; ++i)
        for (int j = 0; j < span; ++j)
            for (int k = 0; k < n2; ++k) {
                const int o[3] = {i - rr, j - rr, k - rr};
                double d2 = 0.0;
                for (int a = 0; a < P.nd; ++a) d2 = d2 + (double)o[a] * (double)o[a];
                if (!(d2 <= r * r)) continue;
                long long lin = 0;
                for (int a = 0; a < P.nd; ++a) {
                    long long p = ((long long)base[a] + o[a]) % P.shape[a];
                    if (p < 0) p += P.shape[a];
                    lin = lin * P.shape[a] + p;
                }
                if (!solid[lin]) {
                    solid[lin] = 1;
                    ++added;
                }
            }
    return added;
}

}  // namespace

extern "C" int64_t prt_pack_balls(uint8_t* solid, int32_t nd, const int32_t* shape,
                                  const double* cand, int64_t ncand, double rmin, double rmax,
                                  double target_frac, int64_t overlap_after, int64_t max_tries,
                                  double* centres, double* radii, int64_t cap, int64_t* state) {
    if (!solid || !shape || !cand || !centres || !radii || !state || (nd != 2 && nd != 3) ||
        ncand < 0 || cap < 0)
        return PRT_E_INVALID;
    Pack P;
    P.nd = nd;
    long long ntot = 1;
    for (int a = 0; a < nd; ++a) {
        if (shape[a] <= 0) return PRT_E_INVALID;
        P.shape[a] = shape[a];
        P.L[a] = (double)shape[a];
        ntot *= shape[a];
        int m = (int)std::floor(P.L[a] / std::fmax(2.0 * rmax, 1e-9));
        P.ncell[a] = m < 1 ? 1 : m;
        P.csize[a] = P.L[a] / P.ncell[a];
    }
    long long nballs = state[0], rejects = state[1], tries = state[2], nsolid = state[3];
    if (nballs > cap) return PRT_E_INVALID;
    for (long long b = 0; b < nballs; ++b) {
        int k[3];
        P.cell_of(centres + b * nd, k);
        P.cells[P.key(k)].push_back((int)b);
    }
    double frac = (double)nsolid / (double)ntot;
    int64_t used = 0;
    while (used < ncand && frac < target_frac && tries < max_tries) {
        const double* u = cand + used * (nd + 1);
        ++used;
        ++tries;
        double c[3] = {0, 0, 0};
        for (int a = 0; a < nd; ++a) c[a] = u[a] * P.L[a];
        const double r = rmin + (rmax - rmin) * u[nd];
        bool ok = true;
        if (rejects < overlap_after && nballs) {
            int k[3];
            P.cell_of(c, k);
            // visit each distinct neighbouring cell once
            std::vector<long long> seen;
            const int n2 = nd == 3 ? 3 : 1;
            for (int i = 0; i < 3 && ok; ++i)
                for (int j = 0; j < 3 && ok; ++j)
                    for (int l = 0; l < n2 && ok; ++l) {
                        const int off[3] = {i - 1, j - 1, l - 1};
                        int kk[3];
                        for (int a = 0; a < nd; ++a)
                            kk[a] = ((k[a] + off[a]) % P.ncell[a] + P.ncell[a]) % P.ncell[a];
                        const long long key = P.key(kk);
                        bool dup = false;
                        for (long long s : seen) dup = dup || s == key;
                        if (dup) continue;
                        seen.push_back(key);
                        auto it = P.cells.find(key);
                        if (it == P.cells.end()) continue;
                        for (int b : it->second)
                            if (!(dist(P, centres + (long long)b * nd, c) >= radii[b] + r)) {
                                ok = false;
                                break;
                            }
                    }
        }
        if (!ok) {
            ++rejects;
            continue;
        }
        if (rejects < overlap_after) rejects = 0;
        if (nballs >= cap) {
            // out of room for centres: give the candidate back
            --used;
            --tries;
            break;
        }
        for (int a = 0; a < nd; ++a) centres[nballs * nd + a] = c[a];
        radii[nballs] = r;
        int k[3];
        P.cell_of(c, k);
        P.cells[P.key(k)].push_back((int)nballs);
        ++nballs;
        nsolid += stamp(P, solid, c, r);
        frac = (double)nsolid / (double)ntot;
    }
    state[0] = nballs;
    state[1] = rejects;
    state[2] = tries;
    state[3] = nsolid;
    return used;
}
