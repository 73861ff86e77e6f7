// march_col.cuh - launch interface of the column-parallel march (deep grids,
// few rays, long marches).
#pragma once

#include "march_common.cuh"

namespace crk {

// Device pointers of one column-parallel march.  The ray columns (f1..f3,
// ksq) use the same [row][32] tile layout as the batched march; the field,
// the factorisation and the workspace of a ray live in the shared memory of
// its cluster.
struct ColArgs {
    const RayDev* rays;
    const int* col_ray;       // rays of this launch, one cluster each
    const EnvDev* envs;
    const double* pool;
    const double2* pd2;       // [ray][set][CR_MAX_NP]
    const int* pd_n;          // [ray][set]
    const double2* pfc;       // partial-fraction residues c_k, [ray][set][CR_MAX_NP]
    const double2* pfcinf;    // c_inf, [ray][set]
    float* f1;
    float* f2;
    float* f3;
    float2* ksq;
    double* tll;
    double2* cpl;
    double* tlg;
    double2* cpg;
    int* flags;
    int compute_grids;
};

// Rows R0..R1 of CTA c of a cluster of C over a column of nz rows.
void col_slice(int nz, int C, int c, int* R0, int* R1);

// Shared memory of one CTA (the largest slice) for a column of nz rows on a
// cluster of `cluster` CTAs with `terms` Pade terms; chosen selects the
// complex64 factor / workspace storage.
size_t col_smem_bytes(int nz, int cluster, int terms, int chosen);

// Smallest cluster whose CTAs hold their slices in shared memory (0: none
// up to 16 CTAs does).
int col_cluster_size(int nz, int terms, int chosen);

// One cluster of `cluster` CTAs of 32 x terms threads per ray; every ray of
// the launch has at most `terms` Pade terms in every set and at most nz_max
// rows.
cudaError_t launch_march_col(const ColArgs& a, int n_rays, int cluster, int terms, int nz_max, int chosen,
                             cudaStream_t st);

// Clusters of the launch's shape that can be resident at once (0: the
// configuration cannot run).
int col_max_active_clusters(int cluster, int terms, int nz_max, int chosen);

}  // namespace crk
