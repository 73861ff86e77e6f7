// march_sum.cuh - launch interface of the partial-fraction (sum form) march.
#pragma once

#include "march_common.cuh"

namespace crk {

// Device pointers of one sum-form march.  Ray columns (f1..f3, ksq, u) and
// lane columns (G and the factors) are stored [row][32] per tile, starting at
// tile_off[t]; ray r of a tile uses index r, lane l of a tile uses index l.
struct SumArgs {
    const RayDev* rays;
    const int* tile_ray;        // [n_tiles * 32]: lane -> ray, -1 unused
    const int* tile_G;          // [n_tiles]: lanes per ray (the tile's largest np)
    const long long* tile_off;  // [n_tiles]
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
    double2 *QD, *AD, *WD, *QU, *AU, *WU;
    double* tll;
    double2* cpl;
    double* tlg;
    double2* cpg;
    int* flags;
    int compute_grids;
};

cudaError_t launch_march_sum(const SumArgs& a, int n_tiles, cudaStream_t st);

}  // namespace crk
