// pipeline_host.h -- the host state and helpers that the C ABI's translation units share:
// pipeline.cu (device contexts, density calls and the entry points), annihilation_host.cu
// (annihilation mode) and query_host.cu (element queries, phase-space samples and the
// persistent element index).  Internal: not part of include/psi_b200.h.
#pragma once
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

#include "psi_b200.h"
#include "psib_kernels.h"

namespace psib {
namespace host {

// the message of the last failure on this thread (psib_last_error)
extern thread_local std::string g_err;
// Record a failure message and return code.
int fail(int code, const char* fmt, ...);

#define CK(x)                                                                                  \
    do {                                                                                       \
        cudaError_t _e = (x);                                                                  \
        if (_e != cudaSuccess)                                                                 \
            return fail(_e == cudaErrorMemoryAllocation ? PSIB_ERR_NOMEM : PSIB_ERR_CUDA,      \
                        "%s failed: %s (%s:%d)", #x, cudaGetErrorString(_e), __FILE__, __LINE__); \
    } while (0)

#define RET(x)                         \
    do {                               \
        int _r = (x);                  \
        if (_r != PSIB_OK) return _r;  \
    } while (0)

// host-memory calls copy the fields out in this many voxel slabs, each beside the update of the next
constexpr int NOUT = 4;

struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
    template <class T> T* as() const { return (T*)p; }
};

// Grow b to at least bytes (contents are not kept).
int ensure(DevBuf& b, size_t bytes);

// The arguments a recorded breadth-first pass depends on.
struct PassKey {
    BfsArgs ba;
    PolyQueue q[3];
    unsigned long long* cq;
    int grid;
};

struct Ctx {
    int device = -1;
    int num_sms = 0;
    cudaStream_t own = nullptr;  // stream of host-memory calls
    cudaStream_t copy = nullptr; // host-memory calls: the field copies, beside the first stages
    cudaEvent_t fields_in = nullptr;
    cudaEvent_t enter = nullptr, leave = nullptr; // device-memory calls: fences with the caller's stream
    cudaStream_t side = nullptr; // atomic mode: the deep-tree images, beside the breadth-first walk
    cudaEvent_t fork = nullptr, join = nullptr;
    cudaEvent_t ev_out[NOUT] = {};
    cudaEvent_t ev[8] = {};
    // host-mode copies
    DevBuf hpos, hvel, hmass, hconn, hfield[6], hgpos, hgmass;
    // items
    DevBuf iframe, ielem, ipid, ikey;
    DevBuf key_sorted, order_in, order;
    DevBuf counts, offsets;
    DevBuf cub_tmp, scratch, scratch_big, iscale;
    DevBuf small; // status, counters, queue heads
    // records
    DevBuf rkey, rmom, rkey_sorted, rperm_in, rperm, rvox, ritem, rmom_sorted, run_vox, run_cnt, run_off;
    // breadth-first clip: three polyhedron queues, the volume histogram, per-level counters, window list
    DevBuf qx[3], qnb[3], qnv[3], qwin[3], qbox[3], qitem[3], hist, bfs_cnt, dfs_list, vsum;
    DevBuf qxd[3]; // the FP64 walk's positions and q
    DevBuf btab, igrid; // batch tables, image -> cutout
    DevBuf adjcoef;     // full adjoint: per-voxel coefficients
    // atomic accumulation: per-voxel sums, tile reference velocities, the mass-correction pass
    DevBuf acc_sum, acc_ref, acc_tsum, acc_vref, acc_toff, fix_list, fix_keys, fix_list_s, fix_keys_s, ifactor;
    DevBuf passes;      // breadth-first pass table
    // annihilation: element tets and boxes, cell registrations, element and tet pairs
    DevBuf a_cnt, a_off, a_ebox, a_tets_a, a_tets_b, a_stats, a_reg_cnt, a_reg_off, a_reg_key, a_reg_elem,
        a_reg_key_s, a_reg_elem_s, a_run_key, a_run_cnt, a_run_off, a_run_lo, a_run_hi, a_pair_cnt, a_pair_off,
        a_pair_key, a_pair_key_s, a_na, a_aoff, a_tp_cnt, a_tp_excl, a_bounds, a_tpairs, a_deep, a_tp_key,
        a_tp_key_s, a_ord_in, a_ord;
    // element queries and phase-space samples
    DevBuf q_in, q_cnt, q_off, q_key, q_key_s, q_out, s_cnt, s_off, s_offs, s_rho, s_vel;
    cudaGraphExec_t pass_exec = nullptr; // one breadth-first pass as a CUDA graph
    PassKey pass_key{};                  // the arguments it was recorded with
    // the capture mode: the sizes a plan call found, and the page-locked copy of the batch tables
    struct Plan {
        bool valid = false;
        long long nelem = 0, nvox = 0, cap_items = 0, ntiles = 0, tiles = 0, qcap = 0;
        int nbatch = 0, max_passes = 0, stride = 0, precision = -1;
        unsigned flags = 0;
        size_t btab_bytes = 0;
    } plan;
    void* btab_host = nullptr;
    size_t btab_host_n = 0;
    std::vector<DevBuf*> all()
    {
        return {&hpos, &hgpos, &hgmass, &hvel, &hmass, &hconn, &hfield[0], &hfield[1], &hfield[2], &hfield[3], &hfield[4],
                &hfield[5], &iframe, &ielem, &ipid, &ikey,
                &key_sorted, &order_in, &order, &counts, &offsets, &cub_tmp, &scratch, &scratch_big, &iscale, &small, &rkey, &rmom,
                &rkey_sorted, &rperm_in, &rperm, &rvox, &ritem, &rmom_sorted, &run_vox, &run_cnt, &run_off,
                &qx[0], &qx[1], &qx[2], &qxd[0], &qxd[1], &qxd[2], &qnb[0], &qnb[1], &qnb[2], &qnv[0], &qnv[1], &qnv[2], &qbox[0], &qbox[1],
                &qbox[2], &qitem[0], &qitem[1], &qitem[2], &hist, &bfs_cnt, &dfs_list, &vsum, &qwin[0], &qwin[1],
                &qwin[2], &btab, &igrid, &passes, &a_cnt, &a_off, &a_ebox, &a_tets_a, &a_tets_b, &a_stats,
                &a_reg_cnt, &a_reg_off, &a_reg_key, &a_reg_elem, &a_reg_key_s, &a_reg_elem_s, &a_run_key,
                &a_run_cnt, &a_run_off, &a_run_lo, &a_run_hi, &a_pair_cnt, &a_pair_off, &a_pair_key,
                &a_pair_key_s, &a_na, &a_aoff, &a_tp_cnt, &a_tp_excl, &a_bounds, &a_tpairs, &a_deep, &a_tp_key,
                &a_tp_key_s, &a_ord_in, &a_ord, &q_in, &q_cnt, &adjcoef, &acc_sum, &acc_ref, &acc_tsum, &acc_vref, &acc_toff,
                &fix_list, &fix_keys, &fix_list_s, &fix_keys_s, &ifactor,
                &q_off, &q_key, &q_key_s, &q_out, &s_cnt, &s_off, &s_offs, &s_rho, &s_vel};
    }
};

// the contexts of devices 0..63, created on first use, under g_mu
extern std::mutex g_mu;
extern Ctx* g_ctx[64];
int get_ctx(int dev, Ctx** out);

// small device block layout (unsigned long long words)
enum { S_STATUS = 0, S_CNT = 1 /* 3 words */, S_TESS = 4 /* 2 */, S_HEAD = 8 /* 4 */, S_RECN = 12, S_NDEEP = 13,
       S_DFS = 14, S_BYTES = 15, S_PASS = 6, S_FIX = 7, S_NMAIN = 16, S_NITEMS = 17, S_WORDS = 18 };

inline size_t round_up(size_t b) { return (b + 15) & ~(size_t)15; }

// An integer from the environment, or dflt when it is unset or empty.
long long env_ll(const char* name, long long dflt);

struct Call {
    const psib_grid* grid;
    const psib_mesh* mesh;
    int mode; // PSIB_MODE_DENSITY or PSIB_MODE_ANNIHILATION
    double reftol;
    int maxlvl;
    int precision;
    int deterministic;
    cudaStream_t st;
    Ctx* C;
    psib_stats* stats;
    // device views
    double* F[6];
    const double *pos, *vel, *mass;
    const int* conn;
    int refine_mode;
    double refine_cell[3];
    long long queue_voxels;
    cudaEvent_t fields_ready; // host-memory calls: recorded when the fields are on the device
    double* const* host_fields; // host-memory calls: where the fields go back (the caller's arrays)
    bool copied_out;          // run_device copied the fields back itself
    // a batch of cutouts (nbatch > 0): host arrays of grids and meshes (device pointers)
    int nbatch;
    const psib_grid* grids;
    const psib_mesh* meshes;
    const double* refine_cell_given;
    int capture;              // options.capture: 0 plain, 1 plan, 2 capture (run_capture)
    int order_cell_bits;      // options.order_cell_bits: coarse cells of the footprint key
    // adjoint call: F[0] holds dL/dm (or adj_coef the full adjoint's per-voxel coefficients);
    // gradients accumulate into these
    bool adjoint;
    double *gpos, *gmass, *gvel;
    const double* adj_coef;
};

// The status word's bits as a PSIB_ERR_* code and message.
int check_status(Call& c, unsigned long long* small_host);
// Device-memory calls run on the library's own stream between these two fences.
int enter_own_stream(Ctx& C, cudaStream_t user);
int leave_own_stream(Ctx& C, cudaStream_t user);
GridDev grid_dev(const psib_grid& g);
MeshDev mesh_dev(const psib_mesh& m, const psib_grid& g, const double* pos, const double* vel, const double* mass,
                 const int* conn, double reftol, const double* lag);
int copy_mesh_in(Call& c, Ctx& C, const psib_mesh& mesh, cudaStream_t st);
int validate_mesh(const psib_mesh* m);
int validate(const psib_grid* g, const psib_mesh* m, int mode, const psib_options* o);
int run_annihilation(Call& c);
int build_cells(Ctx& C, AnnArgs& aa, cudaStream_t st, long long& klaunch, long long& kept);

// Exclusive scan of n counts into n offsets (CUB), on the stream.
template <class In, class Out>
int excl_scan(Ctx& C, const In* in, Out* out, long long n, cudaStream_t st)
{
    if (n >= (1ll << 31)) return fail(PSIB_ERR_OVERFLOW, "a scan of %lld items is too long", n);
    size_t tb = 0;
    CK(cub::DeviceScan::ExclusiveScan(nullptr, tb, in, out, cub::Sum(), (Out)0, (int)n, st));
    RET(ensure(C.cub_tmp, tb));
    CK(cub::DeviceScan::ExclusiveScan(C.cub_tmp.p, tb, in, out, cub::Sum(), (Out)0, (int)n, st));
    return PSIB_OK;
}

// One value from device memory, synchronously.
template <class T>
int read_dev(const T* p, T& out, cudaStream_t st)
{
    CK(cudaMemcpyAsync(&out, p, sizeof(T), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return PSIB_OK;
}

// The bits an index below n needs (at least 1).
inline int bits_for(unsigned long long n)
{
    int b = 1;
    while (b < 64 && (1ull << b) < n) ++b;
    return b;
}

// o[i] = i for i < n.
template <class T>
__global__ void k_iota(T* o, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        o[i] = (T)i;
}

} // namespace host
} // namespace psib
