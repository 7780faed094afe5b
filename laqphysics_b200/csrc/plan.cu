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
#include "hpsi_kinetic.cuh"
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

// Tiles of the kinetic kernel (hpsi_kinetic.cu): row tiles of at most KIN_RELEMS whole
// elements and KIN_ROWS owned nodes, column tiles of KIN_SLOTS slots (<= KIN_NA owned nodes of one
// element each), the first staged node of every tile (the previous element's first node
// when its bridge row is owned) and the staged box extents.  Leaves kin_ok false when an
// element does not fit or the box exceeds the TMA / shared-memory limits.
void build_kinetic(he_plan_host &P, int n)
{
    using namespace he;
    const int ne = P.ne;
    auto esize = [&](int e) { return e + 1 < ne ? P.estart[e + 1] - P.estart[e] + 1 : n - P.estart[e]; };
    auto own = [&](int e) { return (e + 1 < ne ? P.estart[e + 1] : n) - P.estart[e]; };
    P.kin_ok = false;
    P.nodeelem.assign(n, 0);
    for (int e = 0; e < ne; ++e)
        for (int i = P.estart[e]; i < P.estart[e] + own(e); ++i) P.nodeelem[i] = e;
    // transposed planes, rows padded to an even length so that pairs of outputs load as
    // one 16-byte (complex128 plan) or 8-byte (complex64 plan) vector; two entries of
    // padding at the end keep the last pair load inside the array
    P.koff.assign(ne + 1, 0);
    for (int e = 0; e < ne; ++e) P.koff[e + 1] = P.koff[e] + esize(e) * (esize(e) + (esize(e) & 1));
    const size_t total = (size_t)P.koff[ne] + 2;
    P.tre.assign(total, 0.0); P.tim.assign(total, 0.0); P.bre.assign(total, 0.0); P.bim.assign(total, 0.0);
    for (int e = 0; e < ne; ++e) {
        const int m = esize(e), mp = m + (m & 1);
        for (int a = 0; a < m; ++a)
            for (int b = 0; b < m; ++b) {
                const size_t src = 2 * ((size_t)P.eoff[e] + (size_t)a * m + b), dst = (size_t)P.koff[e] + (size_t)b * mp + a;
                P.tre[dst] = P.blocks[src]; P.tim[dst] = P.blocks[src + 1];
                P.bre[dst] = P.bblocks[src]; P.bim[dst] = P.bblocks[src + 1];
            }
    }
    // row tiles
    P.krow.assign(1, 0); P.krbase.clear(); P.krcplx.clear();
    P.kbox_r64 = P.kbox_r32 = P.kbox_c = 0;
    for (int e = 0; e < ne;) {
        int o = 0, f = e;
        while (f < ne && f - e < KIN_RELEMS && o + own(f) <= KIN_ROWS) { o += own(f); ++f; }
        if (f == e) return;
        P.krow.push_back(f);
        e = f;
    }
    P.ntr = (int)P.krow.size() - 1;
    for (int t = 0; t < P.ntr; ++t) {
        const int ea = P.krow[t], eb = P.krow[t + 1];
        const int rb = ea > 0 ? P.estart[ea - 1] : P.estart[ea];
        const int last = eb < ne ? P.estart[eb] : n - 1;
        P.krbase.push_back(rb);
        P.kbox_r64 = std::max(P.kbox_r64, last - rb + 1);
        P.kbox_r32 = std::max(P.kbox_r32, last - (rb & ~1) + 1);
        int cplx = 0;
        for (int e = std::max(ea - 1, 0); e < eb; ++e) cplx |= !P.ereal[e];
        P.krcplx.push_back(cplx);
    }
    P.kbox_r32 += P.kbox_r32 & 1;   // complex64 rows: 8-byte nodes, the box starts and spans 16-byte multiples
    // column slots, packed KIN_SLOTS per tile
    std::vector<int> slots;
    for (int f = 0; f < ne; ++f)
        for (int a0 = 0; a0 < own(f); a0 += KIN_NA) {
            slots.push_back(f); slots.push_back(a0); slots.push_back(std::min(KIN_NA, own(f) - a0));
        }
    const int nslots = (int)slots.size() / 3;
    P.kslot.clear(); P.kcbase.clear();
    for (int s0 = 0; s0 < nslots; s0 += KIN_SLOTS) {
        int first = n, last = 0;
        for (int k = 0; k < KIN_SLOTS; ++k) {
            if (s0 + k < nslots) {
                const int f = slots[3 * (s0 + k)], a0 = slots[3 * (s0 + k) + 1];
                first = std::min(first, (a0 == 0 && f > 0) ? P.estart[f - 1] : P.estart[f]);
                last = std::max(last, std::min(n - 1, P.estart[f] + esize(f) - 1));
                for (int q = 0; q < 3; ++q) P.kslot.push_back(slots[3 * (s0 + k) + q]);
            } else {
                P.kslot.push_back(0); P.kslot.push_back(0); P.kslot.push_back(0);
            }
        }
        P.kcbase.push_back(first);
        P.kbox_c = std::max(P.kbox_c, last - first + 1);
    }
    P.nct = (int)P.kcbase.size();
    const size_t stage = ((size_t)P.kbox_r64 * P.kbox_c * 16 + KIN_STAGE_ALIGN - 1) / KIN_STAGE_ALIGN * KIN_STAGE_ALIGN;
    P.kin_ok = 2 * P.kbox_r64 <= 256 && 2 * P.kbox_r32 <= 256 && P.kbox_c <= 256 &&
               2 * stage + KIN_BRIDGE_BYTES + 64 <= 200 * 1024;
}

// Banded kinetic kernel (hpsi_kinetic.cu): the window and FP64-mma fragments of every
// 8-row group, straight from the CSR (any banded kinetic matrix; no element structure is
// needed), and the staged box of every 64 x 32 tile.  Leaves band_ok false when a window
// exceeds BAND_KS k-steps or the box exceeds the TMA / shared-memory limits.
void build_band(he_plan_host &P, int n, const int *ptr, const int *col, const double *tv, const double *r)
{
    using namespace he;
    P.band_ok = false;
    const int G = (n + BAND_G - 1) / BAND_G;
    P.ngroup = G;
    P.glo.assign(G, 0); P.gks.assign(G, 0); P.greal.assign(G, 3);
    P.gfrag.assign((size_t)G * BAND_KS * 32 * 2, 0.0);
    P.gfragb.assign((size_t)G * BAND_KS * 32 * 2, 0.0);
    for (int g = 0; g < G; ++g) {
        int lo = n, hi = -1;
        for (int i = BAND_G * g; i < std::min(n, BAND_G * (g + 1)); ++i)
            for (int k = ptr[i]; k < ptr[i + 1]; ++k) { lo = std::min(lo, col[k]); hi = std::max(hi, col[k]); }
        if (hi < 0) { lo = std::min(BAND_G * g, n - 1); hi = lo; }
        const int ks = (hi - lo + 4) / 4;
        if (ks > BAND_KS) return;
        P.glo[g] = lo; P.gks[g] = ks;
        for (int i = BAND_G * g; i < std::min(n, BAND_G * (g + 1)); ++i)
            for (int k = ptr[i]; k < ptr[i + 1]; ++k) {
                const int c = col[k], step = (c - lo) / 4, lane = (i - BAND_G * g) * 4 + (c - lo) % 4;
                const size_t idx = 2 * (((size_t)g * BAND_KS + step) * 32 + lane);
                const std::complex<double> T(tv[2 * k], tv[2 * k + 1]);
                const std::complex<double> B = T * (std::complex<double>(r[2 * c], r[2 * c + 1]) -
                                                    std::complex<double>(r[2 * i], r[2 * i + 1]));
                P.gfrag[idx] += T.real(); P.gfrag[idx + 1] += T.imag();
                P.gfragb[idx] += B.real(); P.gfragb[idx + 1] += B.imag();
            }
    }
    for (int g = 0; g < G; ++g)
        for (size_t q = 0; q < (size_t)BAND_KS * 32; ++q) {
            const size_t idx = 2 * ((size_t)g * BAND_KS * 32 + q);
            if (P.gfrag[idx + 1] != 0.0) P.greal[g] &= ~1;
            if (P.gfragb[idx + 1] != 0.0) P.greal[g] &= ~2;
        }
    // tiles: the staged box spans the windows of the tile's groups and the tile itself
    auto span = [&](int first_group, int groups, int extent, int start, int &lo, int &hi) {
        lo = start; hi = start + extent - 1;
        for (int g = first_group; g < std::min(G, first_group + groups); ++g) {
            lo = std::min(lo, P.glo[g]);
            hi = std::max(hi, P.glo[g] + 4 * P.gks[g] - 1);
        }
    };
    P.bntr = (n + BAND_TR - 1) / BAND_TR;
    P.bnct = (n + BAND_TC - 1) / BAND_TC;
    P.brbase.clear(); P.bcbase.clear();
    P.bbox_r64 = P.bbox_r32 = P.bbox_c = 0;
    for (int t = 0; t < P.bntr; ++t) {
        int lo, hi;
        span(t * BAND_WARPS, BAND_WARPS, BAND_TR, t * BAND_TR, lo, hi);
        P.brbase.push_back(lo);
        P.bbox_r64 = std::max(P.bbox_r64, hi - lo + 1);
        P.bbox_r32 = std::max(P.bbox_r32, hi - (lo & ~1) + 1);
    }
    for (int t = 0; t < P.bnct; ++t) {
        int lo, hi;
        span(t * BAND_CG, BAND_CG, BAND_TC, t * BAND_TC, lo, hi);
        P.bcbase.push_back(lo);
        P.bbox_c = std::max(P.bbox_c, hi - lo + 1);
    }
    // row pitch = 4 (mod 8) in nodes: the operand loads of one 8-lane phase hit distinct banks
    auto pad = [](int v) { return v + ((12 - v % 8) % 8); };
    P.bbox_r64 = pad(P.bbox_r64);
    P.bbox_r32 = pad(P.bbox_r32);
    const size_t stage = ((size_t)P.bbox_r64 * P.bbox_c * 16 + KIN_STAGE_ALIGN - 1) / KIN_STAGE_ALIGN * KIN_STAGE_ALIGN;
    const size_t cfrag = (size_t)BAND_CG * BAND_KS * 32 * 16;
    // two stages + the column groups' T and B fragments (B: velocity gauge) + barriers
    P.band_ok = 2 * P.bbox_r64 <= 256 && P.bbox_c <= 256 && 2 * stage + 2 * cfrag + 64 + KIN_STAGE_ALIGN <= 220 * 1024;
}

// Program of the generated channel-mixing kernel.  Each class of channels that share
// Coulomb sources is cut into groups of at most MIXJ_OUT outputs; a group's multipoles are
// ordered by their smallest source and packed into blocks whose sources (at most
// MIXJ_SRC) are loaded once.  In the coupled basis this puts the even multipoles (sources
// in the group's own l1-parity class) and the odd ones (the partner class) in separate
// blocks.
constexpr int MIXJ_OUT = 8, MIXJ_SRC = 8;

void build_mix_program(he_plan_host &P, const std::vector<std::vector<int>> &classes, const int *vptr, const int *vc,
                       const int *vl, const double *vcoef, int nlam, const int *dptr, const int *dc, const int *de)
{
    P.mix.clear();
    for (const auto &cls : classes)
        for (size_t g0 = 0; g0 < cls.size(); g0 += MIXJ_OUT) {
            MixGroup G;
            G.out.assign(cls.begin() + g0, cls.begin() + std::min(cls.size(), g0 + (size_t)MIXJ_OUT));
            // multipoles with edges, each with its sorted source set
            std::vector<std::pair<int, int>> order;   // (smallest source, lambda)
            std::vector<std::set<int>> srcs(nlam);
            for (int d = 0; d < (int)G.out.size(); ++d)
                for (int k = vptr[G.out[d]]; k < vptr[G.out[d] + 1]; ++k) srcs[vl[k]].insert(vc[k]);
            for (int lam = 0; lam < nlam; ++lam)
                if (!srcs[lam].empty()) order.push_back({*srcs[lam].begin(), lam});
            std::sort(order.begin(), order.end());
            MixBlock B;
            std::set<int> bsrc;
            auto close = [&]() {
                if (B.terms.empty()) return;
                B.src.assign(bsrc.begin(), bsrc.end());
                for (auto &T : B.terms)
                    for (auto &si : T.s) si = (int)(std::lower_bound(B.src.begin(), B.src.end(), si) - B.src.begin());
                G.blocks.push_back(B);
                B = MixBlock();
                bsrc.clear();
            };
            for (const auto &o : order) {
                const int lam = o.second;
                std::set<int> merged = bsrc;
                merged.insert(srcs[lam].begin(), srcs[lam].end());
                if ((int)merged.size() > MIXJ_SRC && !B.terms.empty()) { close(); merged = srcs[lam]; }
                bsrc = merged;
                MixTerm T;
                T.lam = lam;
                for (int d = 0; d < (int)G.out.size(); ++d)
                    for (int k = vptr[G.out[d]]; k < vptr[G.out[d] + 1]; ++k)
                        if (vl[k] == lam) { T.d.push_back(d); T.s.push_back(vc[k]); T.w.push_back(vcoef[2 * k]); }
                B.terms.push_back(T);
            }
            close();
            for (int d = 0; d < (int)G.out.size(); ++d)
                for (int k = dptr[G.out[d]]; k < dptr[G.out[d] + 1]; ++k) {
                    const int e = de[k] == 1 ? 0 : 1;
                    G.dd[e].push_back(d); G.ds[e].push_back(dc[k]); G.dk[e].push_back(k);
                }
            P.mix.push_back(G);
        }
}

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
    {
        std::vector<std::vector<int>> cls;
        for (auto &kv : classes) cls.push_back(kv.second);
        build_mix_program(P, cls, vptr, vc, vl, vcoef, nlam, dptr, dc, de);
    }
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
    build_kinetic(P, n);
    build_band(P, n, ptr, col, tv, r);
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
//        11 nodeelem, 12 krow, 13 krbase, 14 krcplx, 15 kslot, 16 kcbase, 17 koff, 18 glo, 19 gks,
//        27 gfrag, 28 gfragb (complex [group][k-step][lane]), 29 greal (bit 0 T, bit 1 B real),
//        32 brbase, 33 bcbase, 34 band scalars {band_ok, ngroup, ntr, nct, box_r64, box_r32, box_c},
//        20 blocks (interleaved complex), 21 bblocks, 22 wcoef, 23 tre, 24 tim, 25 bre, 26 bim,
//        30 scalars {ok, ne, ntile, ng, nlam, maxm, blkmax},
//        31 kinetic scalars {kin_ok, ntr, nct, box_r (complex128), box_r (complex64), box_c}.
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
    case 11: vi = &P.nodeelem; break;
    case 12: vi = &P.krow; break;
    case 13: vi = &P.krbase; break;
    case 14: vi = &P.krcplx; break;
    case 15: vi = &P.kslot; break;
    case 16: vi = &P.kcbase; break;
    case 17: vi = &P.koff; break;
    case 23: vd = &P.tre; break;
    case 24: vd = &P.tim; break;
    case 25: vd = &P.bre; break;
    case 26: vd = &P.bim; break;
    case 18: vi = &P.glo; break;
    case 19: vi = &P.gks; break;
    case 27: vd = &P.gfrag; break;
    case 28: vd = &P.gfragb; break;
    case 29: vi = &P.greal; break;
    case 32: vi = &P.brbase; break;
    case 33: vi = &P.bcbase; break;
    case 34: {
        const int s[7] = {P.band_ok, P.ngroup, P.bntr, P.bnct, P.bbox_r64, P.bbox_r32, P.bbox_c};
        if (dst) memcpy(dst, s, sizeof(s));
        return 7;
    }
    case 31: {
        const int s[6] = {P.kin_ok, P.ntr, P.nct, P.kbox_r64, P.kbox_r32, P.kbox_c};
        if (dst) memcpy(dst, s, sizeof(s));
        return 6;
    }
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
