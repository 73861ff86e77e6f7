// march_sum.cuh - launch interface of the partial-fraction (sum form) march.
#pragma once

#include <cuda.h>  // CUtensorMap

#include "march_common.cuh"

namespace crk {

// Pade terms carried by one lane of the sum-form march.
#ifndef CR_SUM_TERMS
#define CR_SUM_TERMS 2
#endif
constexpr int kT = CR_SUM_TERMS;

// The solve passes stream their rows in blocks of kRB rows, one tensor copy
// per field and block, through a ring of ring_blocks(form) blocks in shared
// memory (complex128 form: CR_SUM_NB; complex64 forms: CR_SUM_NB_C64).
#ifndef CR_SUM_RB
#define CR_SUM_RB 8
#endif
#ifndef CR_SUM_NB
#define CR_SUM_NB 2
#endif
#ifndef CR_SUM_NB_C64
#define CR_SUM_NB_C64 CR_SUM_NB
#endif
constexpr int kRB = CR_SUM_RB;
__host__ __device__ constexpr int ring_blocks(int form) { return form == 0 ? CR_SUM_NB : CR_SUM_NB_C64; }
constexpr int kNBMax = CR_SUM_NB > CR_SUM_NB_C64 ? CR_SUM_NB : CR_SUM_NB_C64;

// Largest lanes-per-ray value the kernels are instantiated for (np <= 10).
constexpr int kMaxP = (10 + kT - 1) / kT;

// Tensor maps of the solve passes' bulk copies (cp.async.bulk.tensor, 2-D,
// 8-byte elements, no multicast).  Every map views one array as rows of the
// 32 columns of a tile ([row][32], as stored) and copies boxes of kRB rows:
//   lane[i]: G, QD, WD, QU, WU - all 32 lane columns of a row;
//   ray[f][P-1]: u, ED, EU, E2 - the floor(32 / P) ray columns of a tile whose
//   rays take P lanes each.
// Row y of a map is element y * 32 of the array; a tile's rows start at
// y = tile_off / 32 (ray arrays) and tile_loff / 32 + t * rows (term slot t of
// the lane arrays).  Rows outside the array read as zeros.
enum { kMapG = 0, kMapQD = 1, kMapWD = 2, kMapQU = 3, kMapWU = 4 };
enum { kMapU = 0, kMapED = 1, kMapEU = 2, kMapE2 = 3 };
struct SumMaps {
    CUtensorMap lane[5];
    CUtensorMap ray[4][kMaxP];
};

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
    int min_p;     // persistent launch: the smallest lanes-per-ray value among the tiles
    SumMaps maps;  // the kernels take SumArgs as a __grid_constant__ parameter
};

// Encodes a.maps for the arrays in a (G, QD, WD, QU, WU over lane_rows rows,
// u, ED, EU and E2 over ray_rows rows; E2 only when not NULL) for the given
// precision form.  Returns false when the driver's encoder is unavailable or
// refuses a map.
bool encode_sum_maps(SumArgs& a, int form, long long ray_rows, long long lane_rows);

// form: an enum cr_precision value.  CR_PLAIN_C128: complex128 factors /
// workspace and FP64 sweeps; CR_CHOSEN_C64R: complex64 factors / workspace
// and FP32 sweeps (the buffers given for G and the factors are then read as
// float2), terms combined in FP64; CR_CHOSEN_C64: as CR_CHOSEN_C64R with the
// couplings (ED / EU read as float2), M u and the term combination in FP32;
// CR_C64_REFINED: as CR_CHOSEN_C64R with one FP64-residual refinement step per
// term and range step (two passes per step; E2 holds the rows' d2).
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

// Loads the kernels (and sets the shared-memory limits) that the two
// launchers above use for these tiles, so that no kernel is loaded at its
// first launch while other streams' kernels run.
cudaError_t prepare_march_sum(const int* tile_P, int n_tiles, int form);

}  // namespace crk
