// Kinetic-energy kernel of H·psi with TMA-staged tiles (hpsi_kinetic.cu).
//
// One CTA works through (row tile, column tile, channel) items.  A row tile is a run of
// whole elements along r1 with at most KIN_ROWS owned nodes; a column tile is up to
// KIN_SLOTS "slots" along r2, a slot being at most KIN_NA owned nodes of one element.
// The staged box holds the tile plus the nodes its bridge rows and columns reach into
// (the previous element), so both kinetic directions read shared memory only.
#pragma once
#include <cuda.h>

#include "common.cuh"

namespace he {

constexpr int KIN_ROWS = 64;                     // owned rows per tile (thread lanes along r1)
constexpr int KIN_SLOTS = 4;                     // column slots per tile
constexpr int KIN_NA = 10;                       // owned columns per slot (outputs per thread)
constexpr int KIN_RELEMS = 8;                    // elements per row tile (bridge rows per tile)
constexpr int KIN_THREADS = KIN_ROWS * KIN_SLOTS;
constexpr int KIN_STAGE_ALIGN = 128;             // byte alignment of each staged box
constexpr int KIN_BRCOLS = KIN_SLOTS * KIN_NA;   // owned columns of a column tile, at most
constexpr int KIN_BRIDGE_BYTES = KIN_RELEMS * KIN_BRCOLS * 16;   // bridge-row partials (complex128)

// Banded formulation on the FP64 tensor cores (mma.sync m8n8k4 f64).  Rows of the
// kinetic matrix are taken in groups of 8; group g couples to the window of nodes
// [glo[g], glo[g] + 4 gks[g]) and its fragment table holds, for k-step s and lane l,
// T[8g + l/4][glo[g] + 4s + l%4] -- the A operand of one direction and the B operand of
// the other, so both electrons accumulate into the same 8x8 output fragments.
constexpr int BAND_G = 8;                        // rows per group (mma M = N = 8)
constexpr int BAND_KS = 8;                       // k-steps per window, at most (window <= 32 nodes)
constexpr int BAND_TR = 64;                      // rows per tile: 8 warps x one row group
constexpr int BAND_TC = 32;                      // columns per tile: 4 column groups
constexpr int BAND_WARPS = BAND_TR / BAND_G;
constexpr int BAND_THREADS = 32 * BAND_WARPS;
constexpr int BAND_CG = BAND_TC / BAND_G;

// Storage precision R (complex128 or complex64 psi); the fragments and the tensor-core
// arithmetic are FP64 in both.
template <typename R> struct BandPlan {
    int n, nc, ngroup, ntr, nct, box_r, box_c;
    int stage_bytes;
    const int *glo, *gks, *greal;                // per group
    const int *brbase, *bcbase;                  // per tile
    const double2 *frag, *fragb;                 // [group][BAND_KS][32]
    int *err;
};

template <typename R> struct KineticPlan {
    int n, nc, ne, ntr, nct, box_r, box_c;
    int stage_bytes;                             // box bytes, rounded up to KIN_STAGE_ALIGN
    const int *estart, *nodeelem, *ereal, *koff;
    const R *tre, *tim, *bre, *bim;              // transposed element blocks (planes, even row stride)
    const int *krow, *krbase, *krcplx;           // row tiles
    const int *kslot, *kcbase;                   // column tiles
    int *err;                                    // device error word (bounded waits that ran out)
};

}  // namespace he
