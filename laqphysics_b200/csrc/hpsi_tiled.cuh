// Tiled H·psi (hpsi_tiled.cu): the radial-stencil kernel and the channel-mixing kernel,
// plus the host-built plan they consume.
#pragma once
#include <vector>

#include "common.cuh"

namespace he {

constexpr int MIX_POINTS = 128;     // points per channel-mixing CTA
constexpr int MIX_GROUP = 4;        // output channels per thread (register block)
constexpr int RAD_ELEMS = 4;        // elements per radial tile and axis
constexpr int RAD_TMAX = 48;        // max owned nodes per radial tile and axis
constexpr int RAD_CHUNK = 8;        // output rows per register chunk

// Device view of the plan.
template <typename R> struct TiledPlan {
    int n, nc, ne, ntile;           // grid size, channels, elements, radial tiles per axis
    const int *estart;              // ne+1 element starts (estart[ne] = n)
    const int *tstart;              // ntile+1 element indices where radial tiles start
    const int *eoff;                // ne+1 offsets of element blocks in `blocks`
    const cplx<R> *blocks;          // per element: dense m x m block T[s+a, s+b], a,b < m
    const cplx<R> *bblocks;         // same layout, B = T (r_b - r_a) (velocity-gauge commutator)
    const int *ereal;               // 1 if the element block is real
    // channel mixing
    int ng, nlam, nwd, nwide;       // groups, multipoles, wide dipole edges, wide Coulomb edges
    const int *gch;                 // ng x MIX_GROUP output channels (-1 = padding)
    const int *wptr;                // ng*nlam+1 wide Coulomb edge offsets, (g, lam) major
    const int *wsrc;                // source channel per wide edge
    const R *wcoef;                 // MIX_GROUP coefficients per wide edge (real)
    const int *dwptr;               // ng+1 wide dipole edge offsets
    const int *dwsrc;               // source channel per wide dipole edge
    const int *dwel;                // electron (1 or 2)
    const int *dwedge;              // MIX_GROUP original dipole edge indices (-1 = none)
};

}  // namespace he

// Channel-mixing program of the generated kernel (jit_mix.cu): output groups (channels
// that share Coulomb sources), each with blocks of multipole terms whose sources are
// loaded once, and the dipole edges per electron.
struct MixTerm {
    int lam = 0;
    std::vector<int> d, s;          // edges: output index in the group, source index in the block
    std::vector<double> w;          // real Coulomb coefficient
};
struct MixBlock {
    std::vector<int> src;           // source channels loaded for the block
    std::vector<MixTerm> terms;
};
struct MixGroup {
    std::vector<int> out;           // output channels
    std::vector<MixBlock> blocks;
    std::vector<int> dd[2], ds[2], dk[2];   // dipole edges per electron: output index, source channel, edge index
};

// Host-owned plan (built by he_create when the tables admit it).
struct he_plan_host {
    bool ok = false;
    std::vector<int> estart, tstart, eoff, ereal, gch, wptr, wsrc, dwptr, dwsrc, dwel, dwedge;
    std::vector<double> blocks, bblocks, wcoef;   // complex as interleaved doubles for blocks
    int ne = 0, ntile = 0, ng = 0, nlam = 0, maxm = 0;
    int blkmax = 0;   // max over tiles and axes of staged block entries (previous row + sum m^2)
    // generated channel-mixing program
    std::vector<MixGroup> mix;
    // banded kinetic kernel (FP64 tensor cores, hpsi_kinetic.cu)
    bool band_ok = false;
    int ngroup = 0, bks = 0, bntr = 0, bnct = 0, bbox_r64 = 0, bbox_r32 = 0, bbox_c = 0;
    std::vector<int> glo, gks, greal;       // per 8-row group: window start, k-steps, T and B real
    std::vector<int> brbase, bcbase;        // per row / column tile: first staged row / column
    std::vector<double> gfrag, gfragb;      // [group][k-step][lane] complex T / B fragments
    // kinetic kernel (TMA-staged tiles, hpsi_kinetic.cu)
    bool kin_ok = false;
    std::vector<int> nodeelem;              // n: element owning each node (a bridge node belongs to the later element)
    std::vector<int> krow, krbase, krcplx;  // row tiles: ntr+1 element starts, first staged row, any complex block
    std::vector<int> kslot, kcbase;         // column tiles: nct x KIN_SLOTS x (element, a0, na), first staged column
    std::vector<int> koff;                  // ne+1 offsets of the transposed blocks
    std::vector<double> tre, tim, bre, bim; // transposed element blocks: [koff[e] + b mp + a] = X[a][b], mp = m + (m & 1)
    int ntr = 0, nct = 0, kbox_r64 = 0, kbox_r32 = 0, kbox_c = 0;
};
