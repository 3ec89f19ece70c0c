// psib_kernels.h -- argument blocks and launchers shared by the translation
// units of libpsi_b200 (host orchestration in pipeline.cu; kernels in
// clip_fp64.cu, clip_mixed.cu, tess.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace psib {

// field presence flags
enum : unsigned { F_X = 1u, F_V = 2u, F_XX = 4u, F_XV = 8u, F_VV = 16u };

// Tet images ("items"), structure of arrays with capacity `cap`:
// vertex v, axis i of item t at p[(3v+i)*cap + t].  Items are written in the
// reference's visiting order (element, refinement path, tet, periodic image).
struct ItemArrays {
    double *p;       // 12 x cap positions (periodic image applied)
    double *u;       // 12 x cap velocities
    double *mass;    // cap
    int *elem;       // cap: element index
    int *pid;        // 4 x cap: particle ids of the 4 vertices (unrefined meshes), else unused
    uint16_t *key;   // cap: ordering key (0 = largest footprint first; 0xFFFF = deep tree)
    long long cap;
};

struct GridDev {
    int n[3];
    double w0[3], w1[3], d[3];
};

struct AccDev {
    double *W, *SX, *SV, *XX, *XV, *VV; // sums, see psib_clip.cuh
    const double *MX, *MV;              // pass-1 voxel means (pass 2)
    unsigned flags;                     // F_* of the requested fields
};

struct ClipArgs {
    ItemArrays it;
    const int *order;        // queue position -> item (may be null: identity)
    long long order_base;    // first queue position of this launch
    long long n;             // queue entries of this launch
    unsigned long long *head;
    GridDev g;
    AccDev acc;
    int pass;                // 1 or 2
    int mom_order;           // polynomial order of the moments (0, 1, 2)
    unsigned *status;
    unsigned long long *counters; // fragments, fragment vertices, splits
    // fragment records (deterministic mode)
    unsigned long long *rec_key;
    double *rec_mom;
    unsigned long long *rec_n;
    unsigned long long rec_cap;
    int rec_nmom;
    long long rec_item_base;
    void *scratch;           // big-tet kernel: NS_BIG slots per thread
};

struct MeshDev {
    int elemtype;
    long long npart, nelem;
    const double *pos, *vel, *mass;
    const int *conn;
    int bdim[3];  // particle lattice of an implicit block mesh
    int edim[3];  // element lattice of an implicit block mesh
    int periodic;
    double box0[3], box1[3];
};

struct TessArgs {
    MeshDev m;
    GridDev g;
    long long e0, e1;          // element range
    int max_lvl;
    double ptol2;
    const long long *offset;   // per element, exclusive (emit)
    long long offset_base;
    int *count;                // per element (count)
    ItemArrays it;
    unsigned *status;
    unsigned long long *counters; // elements kept, tets
};

// ---- launchers (return cudaError_t of the launch) ----
cudaError_t launch_clip_fp64(const ClipArgs &a, bool big, bool record, int grid, int block, cudaStream_t s);
cudaError_t launch_clip_mixed(const ClipArgs &a, bool big, int grid, int block, cudaStream_t s);
size_t scratch_bytes_fp64_big();
size_t scratch_bytes_mixed_big();

cudaError_t launch_tess_count(const TessArgs &a, cudaStream_t s);
cudaError_t launch_tess_emit(const TessArgs &a, cudaStream_t s);

struct FinalArgs {
    GridDev g;
    AccDev acc;
    double *M, *X, *V, *XX, *XV, *VV; // the grid fields (reference layout)
    double *MX, *MV;                  // pass-1 means (written by finalize_means)
    long long nvox;
};
cudaError_t launch_finalize_means(const FinalArgs &f, cudaStream_t s);
cudaError_t launch_finalize_merge(const FinalArgs &f, cudaStream_t s);

struct ApplyArgs {
    const unsigned long long *key; // sorted fragment keys (voxel << 32 | item)
    const double *mom;             // moments, rec_nmom per record, in sorted order
    const unsigned *perm;          // sorted position -> record
    long long nrec;
    int nmom;
    ItemArrays it;
    long long item_base;
    double *M, *X, *V, *XX, *XV, *VV;
};
cudaError_t launch_apply_records(const ApplyArgs &a, cudaStream_t s);

} // namespace psib
