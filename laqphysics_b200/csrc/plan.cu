// Host planner of the tiled H·psi kernels: element structure of the kinetic matrix,
// dense element blocks, radial tiles, output-channel groups and wide edges, plus a
// host-only inspection API used by the CPU tests.
#include <algorithm>
#include <complex>
#include <cstring>
#include <map>
#include <numeric>
#include <set>

#include "common.cuh"
#include "hpsi_tiled.cuh"
#include "operator.cuh"


// =====================================================================================
// Host planning
// =====================================================================================
namespace {

struct UnionFind {
    std::vector<int> p;
    explicit UnionFind(int n) : p(n) { std::iota(p.begin(), p.end(), 0); }
    int find(int x) { while (p[x] != x) x = p[x] = p[p[x]]; return x; }
    void join(int a, int b) { p[find(a)] = find(b); }
};

}  // namespace

// Build the tiled plan from the reference's tables.  Returns false (and the generic
// kernel is used) when the kinetic matrix is not block banded by elements, an element
// is too large for a shared-memory tile, or a Coulomb coefficient is not real.
bool he_build_plan(he_plan_host &P, int n, int nc, const int *ptr, const int *col, const double *tv, int nv,
                   const int *vptr, const int *vc, const int *vl, const double *vcoef, int nlam, int nd,
                   const int *dptr, const int *dc, const int *de, const double *r)
{
    using he::MIX_GROUP;
    P = he_plan_host();
    // --- elements from the first column of each row ---------------------------------
    std::vector<int> first(n), last(n);
    std::set<int> starts;
    for (int i = 0; i < n; ++i) {
        if (ptr[i + 1] == ptr[i]) return false;
        int lo = n, hi = -1;
        for (int k = ptr[i]; k < ptr[i + 1]; ++k) { lo = std::min(lo, col[k]); hi = std::max(hi, col[k]); }
        first[i] = lo; last[i] = hi;
        starts.insert(lo);
    }
    if (!starts.count(0)) return false;
    P.estart.assign(starts.begin(), starts.end());
    const int ne = (int)P.estart.size();
    P.estart.push_back(n);
    P.ne = ne;
    auto esize = [&](int e) { return e + 1 < ne ? P.estart[e + 1] - P.estart[e] + 1 : n - P.estart[e]; };
    // every entry of row i (owned by element e) must lie in element e, or in e-1 for a bridge row
    for (int e = 0; e < ne; ++e) {
        const int s = P.estart[e], m = esize(e);
        if (m > he::RAD_TMAX + 1 || m < 2) return false;
        const int own_end = e + 1 < ne ? P.estart[e + 1] : n;
        for (int i = s; i < own_end; ++i) {
            const int lo_ok = (i == s && e > 0) ? P.estart[e - 1] : s;
            if (first[i] < lo_ok || last[i] > s + m - 1) return false;
        }
    }
    // --- dense element blocks of T and of B = T (r_b - r_a) ---------------------------
    P.eoff.assign(ne + 1, 0);
    for (int e = 0; e < ne; ++e) P.eoff[e + 1] = P.eoff[e] + esize(e) * esize(e);
    P.blocks.assign(2 * (size_t)P.eoff[ne], 0.0);
    P.bblocks.assign(2 * (size_t)P.eoff[ne], 0.0);
    P.ereal.assign(ne, 1);
    for (int e = 0; e < ne; ++e) {
        const int s = P.estart[e], m = esize(e);
        P.maxm = std::max(P.maxm, m);
        for (int a = 0; a < m; ++a) {
            const int i = s + a;
            for (int k = ptr[i]; k < ptr[i + 1]; ++k) {
                const int b = col[k] - s;
                if (b < 0 || b >= m) continue;   // the previous element's part of a bridge row
                const std::complex<double> T(tv[2 * k], tv[2 * k + 1]);
                const std::complex<double> ra(r[2 * i], r[2 * i + 1]), rb(r[2 * col[k]], r[2 * col[k] + 1]);
                const std::complex<double> B = T * (rb - ra);
                const size_t o = 2 * ((size_t)P.eoff[e] + (size_t)a * m + b);
                P.blocks[o] = T.real(); P.blocks[o + 1] = T.imag();
                P.bblocks[o] = B.real(); P.bblocks[o + 1] = B.imag();
                if (T.imag() != 0.0 || B.imag() != 0.0) P.ereal[e] = 0;
            }
        }
    }
    // --- radial tiles: up to RAD_ELEMS elements and RAD_TMAX owned nodes --------------
    P.tstart.push_back(0);
    for (int e = 0; e < ne;) {
        int cnt = 0, own = 0, f = e;
        while (f < ne && cnt < he::RAD_ELEMS) {
            const int o = (f + 1 < ne ? P.estart[f + 1] : n) - P.estart[f];
            if (own + o > he::RAD_TMAX) break;
            own += o; ++cnt; ++f;
        }
        if (cnt == 0) return false;
        e = f;
        P.tstart.push_back(e);
    }
    P.ntile = (int)P.tstart.size() - 1;
    // staged element-block entries of the largest tile axis: previous element's last row + blocks
    for (int k = 0; k < P.ntile; ++k) {
        int entries = P.tstart[k] > 0 ? esize(P.tstart[k] - 1) : 0;
        for (int e = P.tstart[k]; e < P.tstart[k + 1]; ++e) entries += esize(e) * esize(e);
        P.blkmax = std::max(P.blkmax, entries);
    }
    // --- output groups ------------------------------------------------------------------
    // Channels that share Coulomb sources: the connected components of the Coulomb edges
    // (total-L blocks in the coupled basis), split by connectivity through even multipoles
    // (the l1-parity classes: even lambda keeps the parity of l1, odd lambda flips it, so
    // a class sees one parity of sources per lambda).  Each class is cut into groups of
    // MIX_GROUP channels in index order.
    for (int k = 0; k < nv; ++k)
        if (vcoef[2 * k + 1] != 0.0) return false;
    P.nlam = nlam;
    UnionFind component(nc), even(nc);
    for (int c = 0; c < nc; ++c)
        for (int k = vptr[c]; k < vptr[c + 1]; ++k) {
            component.join(c, vc[k]);
            if (vl[k] % 2 == 0) even.join(c, vc[k]);
        }
    std::map<std::pair<int, int>, std::vector<int>> classes;
    for (int c = 0; c < nc; ++c) classes[{component.find(c), even.find(c)}].push_back(c);
    std::vector<std::vector<int>> groups;
    for (auto &kv : classes)
        for (size_t i = 0; i < kv.second.size(); i += MIX_GROUP)
            groups.emplace_back(kv.second.begin() + i,
                                kv.second.begin() + std::min(kv.second.size(), i + (size_t)MIX_GROUP));
    P.ng = (int)groups.size();
    P.gch.assign((size_t)P.ng * MIX_GROUP, -1);
    P.wptr.assign((size_t)P.ng * nlam + 1, 0);
    P.dwptr.assign(P.ng + 1, 0);
    for (int g = 0; g < P.ng; ++g) {
        const auto &grp = groups[g];
        for (int d = 0; d < (int)grp.size(); ++d) P.gch[(size_t)g * MIX_GROUP + d] = grp[d];
        for (int lam = 0; lam < nlam; ++lam) {
            std::map<int, std::vector<double>> wide;
            for (int d = 0; d < (int)grp.size(); ++d)
                for (int k = vptr[grp[d]]; k < vptr[grp[d] + 1]; ++k)
                    if (vl[k] == lam) {
                        auto &w = wide[vc[k]];
                        if (w.empty()) w.assign(MIX_GROUP, 0.0);
                        w[d] += vcoef[2 * k];
                    }
            for (auto &kv : wide) {
                P.wsrc.push_back(kv.first);
                P.wcoef.insert(P.wcoef.end(), kv.second.begin(), kv.second.end());
            }
            P.wptr[(size_t)g * nlam + lam + 1] = (int)P.wsrc.size();
        }
        // dipole edges keyed by (source, electron); repeated keys of one channel open a new slot
        std::vector<std::pair<std::pair<int, int>, std::vector<int>>> dw;
        for (int d = 0; d < (int)grp.size(); ++d)
            for (int k = dptr[grp[d]]; k < dptr[grp[d] + 1]; ++k) {
                bool placed = false;
                for (auto &slot : dw)
                    if (slot.first == std::make_pair(dc[k], de[k]) && slot.second[d] < 0) {
                        slot.second[d] = k; placed = true; break;
                    }
                if (!placed) {
                    std::vector<int> v(MIX_GROUP, -1);
                    v[d] = k;
                    dw.push_back({{dc[k], de[k]}, v});
                }
            }
        for (auto &slot : dw) {
            P.dwsrc.push_back(slot.first.first);
            P.dwel.push_back(slot.first.second);
            P.dwedge.insert(P.dwedge.end(), slot.second.begin(), slot.second.end());
        }
        P.dwptr[g + 1] = (int)P.dwsrc.size();
    }
    (void)nd;
    P.ok = true;
    return true;
}

// ---------------------------------------------------------------------------------
// Planner inspection (host only, no GPU needed): build the plan for a set of tables
// and copy its arrays out, so the tile and group layout can be checked on the CPU.
// ---------------------------------------------------------------------------------
extern "C" void *he_plan_build(int n, int nc, const int *ptr, const int *col, const double *tv, int nv,
                               const int *vptr, const int *vc, const int *vl, const double *vcoef, int nlam, int nd,
                               const int *dptr, const int *dc, const int *de, const double *r)
{
    he_plan_host *P = new he_plan_host();
    he_build_plan(*P, n, nc, ptr, col, tv, nv, vptr, vc, vl, vcoef, nlam, nd, dptr, dc, de, r);
    return P;
}

extern "C" void he_plan_free(void *plan) { delete static_cast<he_plan_host *>(plan); }

// which: 0 estart, 1 tstart, 2 eoff, 3 ereal, 4 gch, 5 wptr, 6 wsrc, 7 dwptr, 8 dwsrc, 9 dwel, 10 dwedge,
//        20 blocks (interleaved complex), 21 bblocks, 22 wcoef, 30 scalars {ok, ne, ntile, ng, nlam, maxm}.
// Returns the element count; copies when dst != NULL.
extern "C" long long he_plan_array(void *plan, int which, void *dst)
{
    const he_plan_host &P = *static_cast<he_plan_host *>(plan);
    const std::vector<int> *vi = nullptr;
    const std::vector<double> *vd = nullptr;
    switch (which) {
    case 0: vi = &P.estart; break;
    case 1: vi = &P.tstart; break;
    case 2: vi = &P.eoff; break;
    case 3: vi = &P.ereal; break;
    case 4: vi = &P.gch; break;
    case 5: vi = &P.wptr; break;
    case 6: vi = &P.wsrc; break;
    case 7: vi = &P.dwptr; break;
    case 8: vi = &P.dwsrc; break;
    case 9: vi = &P.dwel; break;
    case 10: vi = &P.dwedge; break;
    case 20: vd = &P.blocks; break;
    case 21: vd = &P.bblocks; break;
    case 22: vd = &P.wcoef; break;
    case 30: {
        const int s[7] = {P.ok, P.ne, P.ntile, P.ng, P.nlam, P.maxm, P.blkmax};
        if (dst) memcpy(dst, s, sizeof(s));
        return 7;
    }
    default: return -1;
    }
    if (vi) { if (dst) memcpy(dst, vi->data(), vi->size() * sizeof(int)); return (long long)vi->size(); }
    if (dst) memcpy(dst, vd->data(), vd->size() * sizeof(double));
    return (long long)vd->size();
}
