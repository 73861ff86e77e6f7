// march_sum.cuh - launch interface of the partial-fraction (sum form) march.
#pragma once

#include "march_common.cuh"

namespace crk {

// Pade terms carried by one lane of the sum-form march.
#ifndef CR_SUM_TERMS
#define CR_SUM_TERMS 2
#endif
constexpr int kT = CR_SUM_TERMS;

// Device pointers of one sum-form march.  Ray columns (f1..f3, ksq, u) and
// lane columns (G and the factors) are stored [row][32] per tile, starting at
// tile_off[t]; ray r of a tile uses index r, lane l of a tile uses index l.
struct SumArgs {
    const RayDev* rays;
    const int* tile_ray;        // [n_tiles * 32]: lane -> ray, -1 unused
    const int* tile_G;          // [n_tiles]: lanes per ray, ceil(largest np / kT)
    const long long* tile_off;  // [n_tiles]: ray-column base of the tile
    const long long* tile_loff; // [n_tiles]: lane-column base (kT term slots of rows x 32)
    const EnvDev* envs;
    const double* pool;
    const double2* pd1;         // [ray][set][CR_MAX_NP]
    const double2* pd2;
    const int* pd_n;            // [ray][set]
    const double2* pfc;         // partial-fraction residues c_k, [ray][set][CR_MAX_NP]
    const double2* pfcinf;      // c_inf, [ray][set]
    float* f1;
    float* f2;
    float* f3;
    float2* ksq;
    double2* u;
    double2* G;
    double2 *QD, *WD, *QU, *WU;  // lane columns: 1/den and w per term, both directions
    double2 *ED, *EU;            // ray columns: Galerkin coupling into the row (d1 down, d3 up)
    double2* E2;                 // ray columns: the row's d2 (refined form only, else NULL)
    double* tll;
    double2* cpl;
    double* tlg;
    double2* cpg;
    int* flags;
    int compute_grids;
    int tile_begin;             // first tile of this launch (one launch per P)
    // device work queue of the persistent launch: ticket counter (zero at
    // launch), and the n_queue tiles in the order they are taken
    int* ticket;
    const int* queue;
    int n_queue;
    int max_ctas;  // persistent launch: CTAs = every resident slot (0), or this many
};

// form: an enum cr_precision value.  CR_PLAIN_C128: complex128 factors /
// workspace and FP64 sweeps; CR_CHOSEN_C64R: complex64 factors / workspace
// and FP32 sweeps (the buffers given for G and the factors are then read as
// float2), terms combined in FP64; CR_CHOSEN_C64: as CR_CHOSEN_C64R with the
// couplings (ED / EU read as float2), M u and the term combination in FP32;
// CR_C64_REFINED: as CR_CHOSEN_C64R with one FP64-residual refinement step per
// term and range step (two passes per step; E2 holds the rows' d2).
// Largest lanes-per-ray value the kernels are instantiated for (np <= 10).
constexpr int kMaxP = (10 + kT - 1) / kT;
// tile_P: host copy of tile_G.  One launch per run of equal P: run i goes
// on streams[i % n_streams] (independent runs overlap); the number of
// launches is returned in *launches.
// One persistent launch over all n_tiles batched tiles (any mix of P): as many
// CTAs as the device holds at once, each taking tiles from the queue in
// a.queue order by an atomic ticket (a.ticket must read 0 when the launch
// starts).  The number of CTAs launched is returned in *ctas.
cudaError_t launch_march_sum_queue(const SumArgs& a, int n_tiles, int form, cudaStream_t st, int* ctas);

cudaError_t launch_march_sum(const SumArgs& a, const int* tile_P, int n_tiles, int form,
                             const cudaStream_t* streams, int n_streams, int* launches);

}  // namespace crk
