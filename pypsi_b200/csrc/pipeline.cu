// pipeline.cu -- the C ABI (include/psi_b200.h): device contexts, argument
// checks and the host orchestration of one PSI.voxels density call on the GPU
// (annihilation mode and the element queries have theirs in
// annihilation_host.cu and query_host.cu):
//
//   count   elements -> tet images per element             (tess.cu)
//   scan    per-element offsets (CUB)
//   emit    tet images in the reference's visiting order    (tess.cu)
//   order   images sorted by footprint key (CUB radix sort) for load balance
//   clip    mixed precision: the breadth-first walk (bfs.cu), each fragment added to
//           its voxel's sums with FP64 atomics, the sums merged into the fields once;
//           FP64: the depth-first clip (clip_fp64.cu), one record per fragment,
//   sort    records by (voxel, image) (CUB radix sort), and
//   apply   each voxel's records, in image order, with the reference's
//           online field update (tess.cu)
//
// Images are numbered in the reference's visiting order, so each voxel sees
// its fragments in the reference's order and the FP64 path reproduces the
// reference's fields bit for bit.  Meshes whose tet images exceed the item
// budget are streamed in element chunks, in order.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "psi_b200.h"
#include "psib_adjoint.cuh"
#include "psib_device.cuh"
#include "psib_kernels.h"

#include "pipeline_host.h"

using namespace psib;
using namespace psib::host;

namespace psib {
namespace host {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int ensure(DevBuf& b, size_t bytes)
{
    if (bytes == 0) bytes = 16;
    if (b.n >= bytes) return PSIB_OK;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.n = 0;
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        return fail(PSIB_ERR_NOMEM, "cudaMalloc of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    }
    b.n = bytes;
    return PSIB_OK;
}

std::mutex g_mu;
Ctx* g_ctx[64];

int get_ctx(int dev, Ctx** out)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (dev < 0 || dev >= 64) return fail(PSIB_ERR_ARG, "device ordinal %d out of range", dev);
    if (!g_ctx[dev]) {
        Ctx* c = new Ctx();
        c->device = dev;
        CK(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, dev));
        CK(cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&c->fields_in, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->enter, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->leave, cudaEventDisableTiming));
        CK(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming));
        for (auto& e : c->ev_out) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        for (auto& e : c->ev) CK(cudaEventCreate(&e));
        g_ctx[dev] = c;
    }
    *out = g_ctx[dev];
    return PSIB_OK;
}

long long env_ll(const char* name, long long dflt)
{
    const char* s = getenv(name);
    if (!s || !*s) return dflt;
    return atoll(s);
}

int check_status(Call& c, unsigned long long* small_host)
{
    unsigned st = (unsigned)small_host[S_STATUS];
    if (!st) return PSIB_OK;
    if (st & ST_INDEX) return fail(PSIB_ERR_INDEX, "connectivity or voxel index out of range (status 0x%x)", st);
    if (st & (ST_OVERFLOW | ST_DEPTH))
        return fail(PSIB_ERR_OVERFLOW, "a polyhedron outgrew the vertex buffer or slot pool (status 0x%x)", st);
    if (st & ST_GRAPH) return fail(PSIB_ERR_OVERFLOW, "a polyhedron graph walk did not close (status 0x%x)", st);
    return fail(PSIB_ERR_CUDA, "kernel status 0x%x", st);
}

// Device-memory calls run on the library's own non-blocking stream (a CUDA graph cannot be
// recorded on the legacy default stream), after the work already queued on the caller's stream
// and before anything the caller queues next.
int enter_own_stream(Ctx& C, cudaStream_t user)
{
    CK(cudaEventRecord(C.enter, user));
    CK(cudaStreamWaitEvent(C.own, C.enter, 0));
    return PSIB_OK;
}
int leave_own_stream(Ctx& C, cudaStream_t user)
{
    CK(cudaEventRecord(C.leave, C.own));
    CK(cudaStreamWaitEvent(user, C.leave, 0));
    return PSIB_OK;
}

GridDev grid_dev(const psib_grid& g)
{
    GridDev gd;
    for (int i = 0; i < 3; ++i) {
        gd.n[i] = g.n[i];
        gd.w0[i] = g.window[0][i];
        gd.w1[i] = g.window[1][i];
        gd.d[i] = g.d[i];
    }
    return gd;
}

// The device view of a mesh on a grid: arrays, lattice, box, and the
// refinement parameters that depend on the grid (midpoint tolerance) or the
// mesh (Lagrangian cell of the stretch criterion).
MeshDev mesh_dev(const psib_mesh& m, const psib_grid& g, const double* pos, const double* vel, const double* mass,
                 const int* conn, double reftol, const double* lag)
{
    MeshDev md;
    md.elemtype = m.elemtype;
    md.npart = m.npart;
    md.nelem = m.nelem;
    md.pos = pos;
    md.vel = vel;
    md.mass = mass;
    md.conn = conn;
    md.periodic = m.periodic ? 1 : 0;
    for (int i = 0; i < 3; ++i) {
        md.bdim[i] = m.block_dims[i];
        md.edim[i] = m.periodic ? m.block_dims[i] : m.block_dims[i] - 1;
        md.box0[i] = m.box[0][i];
        md.box1[i] = m.box[1][i];
        md.lag[i] = lag ? lag[i] : 0.0;
    }
    double dxmin = 1.0e30;
    for (int i = 0; i < 3; ++i)
        if (g.d[i] < dxmin) dxmin = g.d[i];
    const double tol = reftol * dxmin;
    md.ptol2 = tol * tol;
    return md;
}

// Host-memory calls: copy the mesh to the context's device buffers.
int copy_mesh_in(Call& c, Ctx& C, const psib_mesh& mesh, cudaStream_t st)
{
    const size_t np3 = (size_t)mesh.npart * 3 * sizeof(double);
    RET(ensure(C.hpos, np3));
    CK(cudaMemcpyAsync(C.hpos.p, mesh.pos, np3, cudaMemcpyHostToDevice, st));
    c.pos = C.hpos.as<double>();
    if (mesh.vel) {
        RET(ensure(C.hvel, np3));
        CK(cudaMemcpyAsync(C.hvel.p, mesh.vel, np3, cudaMemcpyHostToDevice, st));
        c.vel = C.hvel.as<double>();
    }
    if (mesh.mass) {
        RET(ensure(C.hmass, (size_t)mesh.nelem * sizeof(double)));
        CK(cudaMemcpyAsync(C.hmass.p, mesh.mass, (size_t)mesh.nelem * sizeof(double), cudaMemcpyHostToDevice, st));
        c.mass = C.hmass.as<double>();
    }
    if (mesh.connectivity) {
        const size_t cb = (size_t)mesh.nelem * mesh.elemtype * sizeof(int);
        RET(ensure(C.hconn, cb));
        CK(cudaMemcpyAsync(C.hconn.p, mesh.connectivity, cb, cudaMemcpyHostToDevice, st));
        c.conn = C.hconn.as<int>();
    }
    return PSIB_OK;
}

int validate_mesh(const psib_mesh* m)
{
    if (!m) return fail(PSIB_ERR_ARG, "mesh is required");
    if (m->elemtype != 4 && m->elemtype != 8 && m->elemtype != 27)
        return fail(PSIB_ERR_ARG, "elemtype must be 4, 8 or 27");
    if (m->nelem < 0 || m->npart < 0) return fail(PSIB_ERR_ARG, "negative mesh size");
    if (m->nelem >= (1ll << 31) || m->npart >= (1ll << 31))
        return fail(PSIB_ERR_ARG, "meshes of 2^31 elements or particles are not supported");
    if (m->nelem > 0 && !m->pos) return fail(PSIB_ERR_ARG, "pos is required");
    if (!m->connectivity) {
        if (m->elemtype != 8) return fail(PSIB_ERR_ARG, "implicit connectivity needs elemtype 8");
        long long np = 1, nel = 1;
        for (int i = 0; i < 3; ++i) {
            if (m->block_dims[i] <= 0) return fail(PSIB_ERR_ARG, "connectivity or block_dims is required");
            np *= m->block_dims[i];
            nel *= m->periodic ? m->block_dims[i] : m->block_dims[i] - 1;
        }
        if (np != m->npart || nel != m->nelem) return fail(PSIB_ERR_ARG, "block_dims disagree with npart/nelem");
    }
    return PSIB_OK;
}

int validate(const psib_grid* g, const psib_mesh* m, int mode, const psib_options* o)
{
    if (!g || !m) return fail(PSIB_ERR_ARG, "grid and mesh are required");
    if (mode != PSIB_MODE_DENSITY && mode != PSIB_MODE_ANNIHILATION) return fail(PSIB_ERR_ARG, "invalid mode %d", mode);
    if (mode == PSIB_MODE_ANNIHILATION && o && o->refine_mode != PSIB_REFINE_MIDPOINT)
        return fail(PSIB_ERR_UNSUPPORTED, "annihilation mode refines by the midpoint criterion only");
    for (int i = 0; i < 3; ++i) {
        if (g->n[i] <= 0) return fail(PSIB_ERR_ARG, "grid n must be positive");
        if (!(g->d[i] > 0.0)) return fail(PSIB_ERR_ARG, "grid cell size d must be positive");
    }
    if ((long long)g->n[0] * g->n[1] * g->n[2] >= (1ll << 32))
        return fail(PSIB_ERR_ARG, "grids of 2^32 voxels or more are not supported");
    if (!g->fields[PSIB_M]) return fail(PSIB_ERR_ARG, "field m is required");
    if (g->fields[PSIB_XX] && !g->fields[PSIB_X]) return fail(PSIB_ERR_ARG, "field 'xx' requires field 'x'");
    if (g->fields[PSIB_XV] && !(g->fields[PSIB_X] && g->fields[PSIB_V]))
        return fail(PSIB_ERR_ARG, "field 'xv' requires fields 'x' and 'v'");
    if (g->fields[PSIB_VV] && !g->fields[PSIB_V]) return fail(PSIB_ERR_ARG, "field 'vv' requires field 'v'");
    RET(validate_mesh(m));
    if (o && o->refine_mode != PSIB_REFINE_MIDPOINT && o->refine_mode != PSIB_REFINE_STRETCH)
        return fail(PSIB_ERR_ARG, "invalid refine_mode %d", o->refine_mode);
    if (o && o->precision != PSIB_FP64 && o->precision != PSIB_MIXED && o->precision != PSIB_FP64_CENTRAL)
        return fail(PSIB_ERR_ARG, "invalid precision %d", o->precision);
    return PSIB_OK;
}

} // namespace host
} // namespace psib

namespace {

// Histogram of the sorted footprint keys: lanes holding equal keys (most of a
// warp, as the keys are sorted) add with one atomic.
__global__ void k_key_hist(const uint16_t* key, long long n, unsigned* hist)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long n32 = (n + 31) / 32 * 32;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n32; i += stride) {
        const bool act = i < n;
        const unsigned k = act ? key[i] : 0x10000u;
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, k);
        if (act && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&hist[k], (unsigned)__popc(peers));
    }
}

__global__ void k_count_deep(const uint16_t* key, long long n, unsigned long long* out)
{
    unsigned long long c = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        c += (key[i] == KEY_DEEP);
    c = __reduce_add_sync(0xFFFFFFFFu, (unsigned)c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

// ---- capture mode: counts and the pass plan on the device ----

// Entries [*total, cap) of a fixed-size item buffer hold no image: their key sorts last.
__global__ void k_pad_keys(uint16_t* key, const long long* total, long long cap)
{
    const long long t0 = *total;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cap; i += (long long)gridDim.x * blockDim.x)
        if (i >= t0) key[i] = (uint16_t)KEY_PAD;
}

// Counts of the main images (key < KEY_DEEP) and the deep-tree kernel's (KEY_DEEP) among cap keys;
// sorted, they are [0, nmain) and [nmain, nmain + ndeep).  The two words start at zero.
__global__ void k_key_classes(const uint16_t* key, long long cap, unsigned long long* nmain, unsigned long long* ndeep)
{
    unsigned m = 0, d = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cap; i += (long long)gridDim.x * blockDim.x) {
        const unsigned k = key[i];
        m += k < KEY_DEEP;
        d += k == KEY_DEEP;
    }
    m = __reduce_add_sync(0xFFFFFFFFu, m);
    d = __reduce_add_sync(0xFFFFFFFFu, d);
    if ((threadIdx.x & 31) == 0) {
        if (m) atomicAdd(nmain, (unsigned long long)m);
        if (d) atomicAdd(ndeep, (unsigned long long)d);
    }
}

// Histogram of the volume classes (key >> KEY_CELL_BITS) of the first *n sorted keys (n on the
// device).  The keys sort by class first, so the classes give the passes as the keys would.
__global__ void k_key_hist_dev(const uint16_t* key, const unsigned long long* n_dev, unsigned* hist)
{
    const long long n = (long long)*n_dev;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long n32 = (n + 31) / 32 * 32;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n32; i += stride) {
        const bool act = i < n;
        const unsigned k = act ? (unsigned)key[i] >> KEY_CELL_BITS : 0x10000u;
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, k);
        if (act && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&hist[k], (unsigned)__popc(peers));
    }
}

// The host planner of bfs_clip on one thread: images in key order, a pass takes images while the
// sum of their box volumes stays within cap.  hist counts the volume classes of the main images;
// passes[0..max_passes] (unused passes empty at nmain).
__global__ void k_plan_passes(const unsigned* hist, long long cap, long long* passes, int max_passes,
                              const unsigned long long* nmain, unsigned* status)
{
    if (blockIdx.x || threadIdx.x) return;
    const long long n = (long long)*nmain;
    int p = 0;
    long long cur = 0, pos = 0;
    passes[0] = 0;
    for (int k = 0; k < (int)(KEY_DEEP >> KEY_CELL_BITS); ++k) {
        long long cnt = hist[k];
        const long long vol = key_volume((unsigned)k << KEY_CELL_BITS);
        while (cnt > 0) {
            long long take = (cap - cur) / vol;
            if (take > cnt) take = cnt;
            if (take == 0) {
                if (cur == 0 || p + 1 >= max_passes) { // one image above the capacity, or too many passes
                    atomicOr(status, ST_OVERFLOW);
                    for (int q = p + 1; q <= max_passes; ++q) passes[q] = n;
                    return;
                }
                passes[++p] = pos;
                cur = 0;
                continue;
            }
            cur += take * vol;
            pos += take;
            cnt -= take;
        }
    }
    for (int q = p + 1; q <= max_passes; ++q) passes[q] = n;
}

// The correction pass: one pass over the listed images, whose box volumes must fit the queues.
__global__ void k_plan_list(const uint16_t* keys, const unsigned long long* n_dev, long long cap, long long* passes,
                            int max_passes, unsigned* status)
{
    const long long n = (long long)*n_dev;
    long long vol = 0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) vol += key_volume(keys[i]);
    __shared__ unsigned long long sum;
    if (threadIdx.x == 0) sum = 0;
    __syncthreads();
    atomicAdd(&sum, (unsigned long long)vol);
    __syncthreads();
    if (threadIdx.x == 0) {
        if ((long long)sum > cap) atomicOr(status, ST_OVERFLOW);
        passes[0] = 0;
        for (int q = 1; q <= max_passes; ++q) passes[q] = n;
    }
}

// Bits of the footprint key's coarse cell per axis: b bits shared out x, y, z, x, ...
// (0 means the default 7 = 8 x 4 x 4 cells; negative means no spatial order).
void order_cells(int b, int* cb)
{
    cb[0] = cb[1] = cb[2] = 0;
    if (b == 0) b = KEY_CELL_BITS;
    if (b < 0) return;
    if (b > KEY_CELL_BITS) b = KEY_CELL_BITS;
    for (int i = 0; i < b; ++i) ++cb[i % 3];
}

// levels of one breadth-first pass: the bisection (at most DMAX_MAIN cuts) and up to 6 window planes
constexpr int NLEV = DMAX_MAIN + 6;
// per pass: level-queue counts [0, NLEV], leaf-queue counts [NLEV + 1, 2 NLEV + 1], the leaf
// queues' high-end counts [2 NLEV + 2, 3 NLEV + 2] and the level queues' [3 NLEV + 3, 4 NLEV + 3]
constexpr int NCNT = 4 * NLEV + 4;

// One breadth-first pass: reset the per-level counts, then init, leaf, and NLEV x (level, leaf),
// then advance the pass counter.  The pass it walks is read from the device pass table.
cudaError_t bfs_pass(const BfsArgs& ba, const PolyQueue* Q, unsigned long long* cq, int grid, cudaStream_t s)
{
    unsigned long long* cl = cq + NLEV + 1;
    unsigned long long* ch = cq + 2 * NLEV + 2;
    unsigned long long* cqh = cq + 3 * NLEV + 3;
    cudaError_t e = cudaMemsetAsync(cq, 0, NCNT * sizeof(unsigned long long), s);
    BfsArgs b = ba;
    b.out = Q[0];
    b.out.count = &cq[0];
    b.out.count_hi = &cqh[0];
    b.leaf = Q[2];
    b.leaf.count = &cl[0];
    b.leaf.count_hi = &ch[0];
    auto init = ba.fp64 ? launch_bfs64_init : launch_bfs_init;
    auto level = ba.fp64 ? launch_bfs64_level : launch_bfs_level;
    auto leaf = ba.fp64 ? launch_bfs64_leaf : launch_bfs_leaf;
    if (e == cudaSuccess) e = init(b, grid, s);
    if (e == cudaSuccess) e = leaf(b, grid, s);
    int ia = 0;
    for (int lvl = 0; lvl < NLEV && e == cudaSuccess; ++lvl) {
        b.in = Q[ia];
        b.in.count = &cq[lvl];
        b.in.count_hi = &cqh[lvl];
        b.out = Q[1 - ia];
        b.out.count = &cq[lvl + 1];
        b.out.count_hi = &cqh[lvl + 1];
        b.leaf.count = &cl[lvl + 1];
        b.leaf.count_hi = &ch[lvl + 1];
        b.last = lvl == NLEV - 1;
        e = level(b, grid, s);
        if (e == cudaSuccess) e = leaf(b, grid, s);
        ia = 1 - ia;
    }
    if (e == cudaSuccess) e = launch_bfs_advance(b, s);
    return e;
}

// The queue capacity (in 32-wide tiles) and pass count a breadth-first walk used; the capture
// mode sizes its fixed launch sequence from them.
struct BfsSizes {
    long long tiles = 0, cap = 0, npass = 0;
};

// Clip of queue positions [0, nmain) by the breadth-first walk: mixed precision (bfs.cu; images
// that need the window clip come back in a list for the depth-first kernel when PSIB_BFS_WINDOW=0)
// or, with fp64, the bit-exact FP64 walk (bfs_fp64.cu, raw records; window planes cut in the walk).
// Images are sorted by index-box volume, largest first; a pass takes images while the sum of
// their box volumes -- a bound on every queue of the pass -- stays within the queue capacity.
// keys: the footprint keys of the queue positions [0, nmain), ascending.
int bfs_clip(Ctx& C, ClipArgs& ca, long long nmain, long long nitems, unsigned long long* sm, int clip_grid,
             int clip_block, long long queue_voxels, bool batch, cudaStream_t st, long long& launches,
             long long& klaunch, const uint16_t* keys, BfsSizes* sizes = nullptr, bool fp64 = false)
{
    // bytes of one queue element's positions (FP32, or FP64 position and q)
    const size_t xbytes = fp64 ? (size_t)MAXV * 6 * sizeof(double) : (size_t)MAXV * 3 * sizeof(float);
    DevBuf* qxb = fp64 ? C.qxd : C.qx;
    RET(ensure(C.hist, 65536 * sizeof(unsigned)));
    CK(cudaMemsetAsync(C.hist.p, 0, 65536 * sizeof(unsigned), st));
    k_key_hist<<<C.num_sms * 4, 256, 0, st>>>(keys, nmain, C.hist.as<unsigned>());
    CK(cudaGetLastError());
    klaunch++;
    std::vector<unsigned> hist(65536);
    CK(cudaMemcpyAsync(hist.data(), C.hist.p, 65536 * sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    // queue capacity in box voxels: asked for, or up to 64M within 35% of the free memory
    // (three queues of bytes_per_elem each)
    long long cap = queue_voxels;
    if (cap <= 0) {
        const long long bytes_per_elem = (long long)xbytes + MAXV * 4 + 1 + 1 + 12 + 4;
        size_t freeb = 0, totalb = 0;
        if (cudaMemGetInfo(&freeb, &totalb) != cudaSuccess) {
            cudaGetLastError();
            freeb = 0;
        }
        long long have = (long long)(qxb[0].n / xbytes); // queues already allocated count as free
        cap = std::max<long long>(have, (long long)(0.35 * (double)freeb) / (3 * bytes_per_elem));
        cap = std::min<long long>(cap, 64ll << 20);
    }
    cap = std::max<long long>(env_ll("PSIB_BFS_CAP", cap), 1024);
    std::vector<long long> qb{0};
    long long cur = 0, pos = 0;
    for (int k = 0; k < (int)KEY_DEEP; ++k) {
        long long cnt = hist[k];
        const long long vol = key_volume((unsigned)k);
        while (cnt > 0) {
            const long long take = std::min(cnt, (cap - cur) / vol);
            if (take == 0) {
                qb.push_back(pos);
                cur = 0;
                continue;
            }
            cur += take * vol;
            pos += take;
            cnt -= take;
        }
    }
    if (qb.back() != pos) qb.push_back(pos);
    if (pos != nmain) return fail(PSIB_ERR_CUDA, "footprint histogram covers %lld of %lld images", pos, nmain);
    // the largest pass bounds every queue
    long long need = 0;
    {
        size_t p = 0;
        long long acc = 0, at = 0;
        for (int k = 0; k < (int)KEY_DEEP && p + 1 < qb.size(); ++k) {
            const long long vol = key_volume((unsigned)k);
            for (long long cnt = hist[k]; cnt > 0;) {
                const long long take = std::min(cnt, qb[p + 1] - at);
                acc += take * vol;
                at += take;
                cnt -= take;
                if (at == qb[p + 1]) {
                    need = std::max(need, acc);
                    acc = 0;
                    if (++p + 1 >= qb.size()) break;
                }
            }
        }
    }
    const size_t tiles = (size_t)(std::max<long long>(std::min(need, cap), 32) + 31) / 32;
    PolyQueue Q[3];
    for (int i = 0; i < 3; ++i) {
        RET(ensure(qxb[i], tiles * 32 * xbytes));
        RET(ensure(C.qnb[i], tiles * 32 * MAXV * sizeof(uint32_t)));
        RET(ensure(C.qnv[i], tiles * 32));
        RET(ensure(C.qwin[i], tiles * 32));
        RET(ensure(C.qbox[i], tiles * 32 * 3 * sizeof(uint32_t)));
        RET(ensure(C.qitem[i], tiles * 32 * sizeof(uint32_t)));
        Q[i] = PolyQueue{fp64 ? nullptr : C.qx[i].as<float>(), C.qnb[i].as<uint32_t>(), C.qnv[i].as<uint8_t>(),
                         C.qwin[i].as<uint8_t>(), C.qbox[i].as<uint32_t>(), C.qitem[i].as<uint32_t>(), nullptr,
                         (unsigned long long)tiles * 32};
        Q[i].xq = fp64 ? C.qxd[i].as<double>() : nullptr;
    }
    RET(ensure(C.dfs_list, (size_t)std::max<long long>(nmain, 1) * sizeof(int)));
    RET(ensure(C.bfs_cnt, NCNT * sizeof(unsigned long long)));
    unsigned long long* cq = C.bfs_cnt.as<unsigned long long>();
    CK(cudaMemsetAsync(&sm[S_DFS], 0, 8, st));

    BfsArgs ba = {};
    ba.c = ca;
    ba.dfs_list = C.dfs_list.as<int>();
    ba.dfs_count = &sm[S_DFS];
    ba.bytes = &sm[S_BYTES];
    ba.window_bfs = env_ll("PSIB_BFS_WINDOW", 1) != 0;
    ba.fp64 = fp64 ? 1 : 0;
    // Fewer resident level blocks than fit (PSIB_LEVEL_BLOCKS=6, the freed shared memory given to L1)
    // measured within noise of all that fit (64^3 -> 128^3 clip 43.5 against 42.6 ms, three runs each)
    ba.level_blocks = (int)env_ll("PSIB_LEVEL_BLOCKS", 0);
    ba.leaf_split = fp64 ? 0 : (int)env_ll("PSIB_LEAF_SPLIT", 7);
    // the level queues filled from both ends too (PSIB_LEVEL_SPLIT=7): the level launches alone
    // 10 % faster, but whole steps measured 4 % slower and more variable, so off by default
    ba.level_split = fp64 ? 0 : (int)env_ll("PSIB_LEVEL_SPLIT", 0);
    // fewer level blocks leave shared memory unused: give it to L1 (one block is 30 KB of 228)
    if (!fp64) bfs_level_carveout(ba.level_blocks > 0 ? std::min(100, (ba.level_blocks * 31 * 100 + 227) / 228) : 0);
    RET(ensure(C.vsum, (size_t)std::max<long long>(nitems, 1) * sizeof(double)));
    ba.vsum = C.vsum.as<double>();
    // the pass table on the device; a device counter picks the pass, so every pass runs
    // the same launches
    const long long npass = (long long)qb.size() - 1;
    RET(ensure(C.passes, qb.size() * sizeof(long long)));
    CK(cudaMemcpyAsync(C.passes.p, qb.data(), qb.size() * sizeof(long long), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(&sm[S_PASS], 0, 8, st));
    ba.passes = C.passes.as<long long>();
    ba.pass_idx = &sm[S_PASS];
    const int grid = C.num_sms;
    bfs_prepare();
    bfs64_prepare();
    // One pass: reset the per-level counts, then init, leaf, and NLEV x (level, leaf), then
    // advance the pass counter.  Batches record it once as a CUDA graph and replay it for every
    // pass (and in later calls whose arguments are the same); plain launches if the graph cannot
    // be made.  Single calls launch directly: measured at 128^3 -> 256^3 the replay was 3 %
    // slower, and for 512 cutouts no faster (PSIB_BFS_GRAPH=0/1 overrides).
    auto pass = [&](cudaStream_t s) -> cudaError_t { return bfs_pass(ba, Q, cq, grid, s); };
    bool graphed = false;
    if (env_ll("PSIB_BFS_GRAPH", batch ? 1 : 0) != 0) {
        PassKey key{};
        key.ba = ba;
        key.ba.c.n = 0; // depth-first fields the walk does not read
        key.ba.c.order_base = 0;
        key.ba.c.head = nullptr;
        key.ba.c.scratch = nullptr;
        for (int i = 0; i < 3; ++i) key.q[i] = Q[i];
        key.cq = cq;
        key.grid = grid;
        if (!C.pass_exec || memcmp(&key, &C.pass_key, sizeof(key)) != 0) {
            if (C.pass_exec) cudaGraphExecDestroy(C.pass_exec);
            C.pass_exec = nullptr;
            cudaGraph_t gph = nullptr;
            if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                const cudaError_t e = pass(st);
                const cudaError_t e2 = cudaStreamEndCapture(st, &gph);
                if (e == cudaSuccess && e2 == cudaSuccess && gph &&
                    cudaGraphInstantiate(&C.pass_exec, gph, 0) == cudaSuccess) {
                    C.pass_key = key;
                } else {
                    C.pass_exec = nullptr;
                }
                if (gph) cudaGraphDestroy(gph);
            }
            cudaGetLastError(); // a failed capture falls back to plain launches
        }
        if (C.pass_exec) {
            for (long long p = 0; p < npass; ++p) CK(cudaGraphLaunch(C.pass_exec, st));
            graphed = true;
        }
    }
    if (!graphed)
        for (long long p = 0; p < npass; ++p) CK(pass(st));
    klaunch += (3 + 2 * NLEV) * npass;
    launches += (2 + 2 * NLEV) * npass;
    if (sizes) {
        sizes->tiles = (long long)tiles;
        sizes->cap = cap;
        sizes->npass = npass;
    }
    if (!fp64) { // the FP64 walk's images need no mass correction
        CK(launch_bfs_finalize(ba, nitems, C.num_sms, st));
        klaunch++;
    }
    unsigned long long ndfs = 0;
    CK(cudaMemcpyAsync(&ndfs, &sm[S_DFS], 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (ndfs > 0) {
        ClipArgs cw = ca;
        cw.order = C.dfs_list.as<int>();
        cw.order_base = 0;
        cw.n = (long long)ndfs;
        cw.head = &sm[S_HEAD];
        if (fp64) CK(launch_clip_fp64(cw, false, clip_grid, clip_block, st));
        else CK(launch_clip_mixed(cw, false, false, clip_grid, clip_block, st));
        launches++;
    }
    return PSIB_OK;
}

// the Lagrangian cell of the stretch criterion: given, or box / block_dims of a periodic block mesh
int stretch_cell(const psib_mesh& m, const double* given, double* lag)
{
    const bool ok = given && given[0] > 0.0 && given[1] > 0.0 && given[2] > 0.0;
    for (int i = 0; i < 3; ++i) {
        if (ok) lag[i] = given[i];
        else if (m.periodic && m.block_dims[i] > 0) lag[i] = (m.box[1][i] - m.box[0][i]) / m.block_dims[i];
        else return fail(PSIB_ERR_ARG, "the stretch criterion needs refine_cell or a periodic block mesh");
    }
    return PSIB_OK;
}

// The mass correction of the atomic mode.  A breadth-first image's FP32 walk
// can miss the exact q-volume by O(1e-7) where a fragment vertex falls back to
// its FP32 position; the record path scales every fragment of such an image by
// target / (sum of its fragment volumes) when it applies the records.  Atomic
// sums are linear in an image's mass, so the same correction is a second walk
// of just those images with mass factor (scale - 1): bfs_finalize has computed
// scale for every image; those more than tol from 1 are listed (footprint keys
// ascending, as the pass planner wants them) and walked again.
int correct_masses(Ctx& C, const ClipArgs& ca, long long nitems, unsigned long long* sm, int clip_grid,
                   int clip_block, long long queue_voxels, cudaStream_t st, long long& launches, long long& klaunch,
                   long long& ncorr)
{
    constexpr double tol = 1e-14;
    RET(ensure(C.fix_list, (size_t)nitems * sizeof(int)));
    RET(ensure(C.fix_keys, (size_t)nitems * sizeof(uint16_t)));
    RET(ensure(C.ifactor, (size_t)nitems * sizeof(double)));
    CK(cudaMemsetAsync(&sm[S_FIX], 0, 8, st));
    CK(launch_correction_select(ca.it, ca.scale, nitems, tol, C.fix_list.as<int>(), C.fix_keys.as<uint16_t>(),
                                C.ifactor.as<double>(), &sm[S_FIX], C.num_sms, st));
    klaunch++;
    unsigned long long n = 0;
    CK(cudaMemcpyAsync(&n, &sm[S_FIX], 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    ncorr = (long long)n;
    if (n == 0) return PSIB_OK;
    RET(ensure(C.fix_list_s, (size_t)n * sizeof(int)));
    RET(ensure(C.fix_keys_s, (size_t)n * sizeof(uint16_t)));
    size_t tb = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, C.fix_keys.as<uint16_t>(), C.fix_keys_s.as<uint16_t>(),
                                       C.fix_list.as<int>(), C.fix_list_s.as<int>(), (int)n, 0, 16, st));
    RET(ensure(C.cub_tmp, tb));
    CK(cub::DeviceRadixSort::SortPairs(C.cub_tmp.p, tb, C.fix_keys.as<uint16_t>(), C.fix_keys_s.as<uint16_t>(),
                                       C.fix_list.as<int>(), C.fix_list_s.as<int>(), (int)n, 0, 16, st));
    ClipArgs cf = ca;
    cf.order = C.fix_list_s.as<int>();
    cf.acc.factor = C.ifactor.as<double>();
    return bfs_clip(C, cf, (long long)n, nitems, sm, clip_grid, clip_block, queue_voxels, false, st, launches,
                    klaunch, C.fix_keys_s.as<uint16_t>());
}

// The batch tables a batch call's kernels read: every cutout's mesh and grid, the element and
// voxel offsets, and the field pointers, laid out in one host buffer.
struct BatchTables {
    std::vector<char> h;
    size_t o_mesh = 0, o_grid = 0, o_eoff = 0, o_voff = 0, o_fptr = 0;
};
int batch_tables(const Call& c, const std::vector<long long>& eoff, const std::vector<unsigned long long>& voff,
                 BatchTables& t)
{
    const int nb = c.nbatch;
    t.o_mesh = 0;
    t.o_grid = round_up(t.o_mesh + nb * sizeof(MeshDev));
    t.o_eoff = round_up(t.o_grid + nb * sizeof(GridDev));
    t.o_voff = round_up(t.o_eoff + (nb + 1) * 8);
    t.o_fptr = round_up(t.o_voff + (nb + 1) * 8);
    t.h.assign(round_up(t.o_fptr + 6 * nb * sizeof(double*)), 0);
    for (int b = 0; b < nb; ++b) {
        const psib_mesh& mb = c.meshes[b];
        double lag[3] = {0.0, 0.0, 0.0};
        if (c.refine_mode == PSIB_REFINE_STRETCH) RET(stretch_cell(mb, c.refine_cell_given, lag));
        ((MeshDev*)(t.h.data() + t.o_mesh))[b] =
            mesh_dev(mb, c.grids[b], mb.pos, mb.vel, mb.mass, mb.connectivity, c.reftol, lag);
        ((GridDev*)(t.h.data() + t.o_grid))[b] = grid_dev(c.grids[b]);
        for (int f = 0; f < 6; ++f) ((double**)(t.h.data() + t.o_fptr))[6 * b + f] = c.grids[b].fields[f];
    }
    memcpy(t.h.data() + t.o_eoff, eoff.data(), (nb + 1) * 8);
    memcpy(t.h.data() + t.o_voff, voff.data(), (nb + 1) * 8);
    return PSIB_OK;
}

int run_device(Call& c)
{
    if (c.mode == PSIB_MODE_ANNIHILATION) return run_annihilation(c);
    Ctx& C = *c.C;
    const psib_grid& g = *c.grid;
    const psib_mesh& m = *c.mesh;
    cudaStream_t st = c.st;
    const bool batch = c.nbatch > 0;
    long long nvox = (long long)g.n[0] * g.n[1] * g.n[2];
    long long ne = m.nelem;
    std::vector<long long> eoff{0};
    std::vector<unsigned long long> voff{0};
    if (batch) {
        for (int b = 0; b < c.nbatch; ++b) {
            const psib_grid& gb = c.grids[b];
            eoff.push_back(eoff.back() + c.meshes[b].nelem);
            voff.push_back(voff.back() + (unsigned long long)gb.n[0] * gb.n[1] * gb.n[2]);
        }
        nvox = (long long)voff.back();
        ne = eoff.back();
    }

    unsigned flags = 0;
    if (c.F[1]) flags |= F_X;
    if (c.F[2]) flags |= F_V;
    if (c.F[3]) flags |= F_XX;
    if (c.F[4]) flags |= F_XV;
    if (c.F[5]) flags |= F_VV;
    const int order = (flags & (F_XX | F_XV | F_VV)) ? 2 : (flags & (F_X | F_V)) ? 1 : 0;
    const bool mixed = c.precision == PSIB_MIXED && !c.adjoint;
    // central-form records: the mixed kernel, or the FP64 walk in PSIB_FP64_CENTRAL
    const bool central = (mixed || c.precision == PSIB_FP64_CENTRAL) && !c.adjoint;
    // the mixed kernel walks the main images breadth first (PSIB_BFS=0: depth first)
    bool use_bfs = mixed && env_ll("PSIB_BFS", 1) != 0;
    // the bit-exact FP64 mode walks them breadth first too (PSIB_BFS64=0: depth first)
    bool use_bfs64 = c.precision == PSIB_FP64 && !c.adjoint && env_ll("PSIB_BFS64", 1) != 0;
    for (int b = 0; b < (batch ? c.nbatch : 1); ++b)
        for (int i = 0; i < 3; ++i)
            if ((batch ? c.grids[b] : g).n[i] >= 0xFFFF) use_bfs = use_bfs64 = false; // box bounds: 16 bits
    // 1, 4 or 10 moments per record (FP32 kernel: m0, q-centroid, central second moment)
    const int nmom = order == 2 ? 10 : order == 1 ? 4 : 1;
    // Fragments added to per-voxel sums with atomics (deterministic == 0): central-form
    // fragments whose mass correction is 1 or applied by a second walk -- the breadth-first
    // walk (window images included) and the FP64 walks.  Otherwise records, sorted and applied.
    const bool window_bfs = env_ll("PSIB_BFS_WINDOW", 1) != 0;
    const bool atomic = central && !c.deterministic && !c.adjoint && (!mixed || (use_bfs && window_bfs));

    const GridDev gd = grid_dev(g);
    const MeshDev md = mesh_dev(m, g, c.pos, c.vel, c.mass, c.conn, c.reftol, c.refine_cell);
    // a batch: per-cutout meshes and grids, element and voxel offsets, field pointers
    const MeshDev* d_meshes = nullptr;
    const GridDev* d_grids = nullptr;
    const long long* d_eoff = nullptr;
    const unsigned long long* d_voff = nullptr;
    double* const* d_fptr = nullptr;
    if (batch) {
        BatchTables bt;
        RET(batch_tables(c, eoff, voff, bt));
        RET(ensure(C.btab, bt.h.size()));
        CK(cudaMemcpyAsync(C.btab.p, bt.h.data(), bt.h.size(), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st)); // the host copy goes out of scope
        if (c.capture == 1) {
            // a page-locked copy for the capture calls, which may not allocate
            if (C.btab_host_n < bt.h.size()) {
                if (C.btab_host) cudaFreeHost(C.btab_host);
                C.btab_host = nullptr;
                C.btab_host_n = 0;
                CK(cudaMallocHost(&C.btab_host, bt.h.size()));
                C.btab_host_n = bt.h.size();
            }
        }
        d_meshes = (const MeshDev*)(C.btab.as<char>() + bt.o_mesh);
        d_grids = (const GridDev*)(C.btab.as<char>() + bt.o_grid);
        d_eoff = (const long long*)(C.btab.as<char>() + bt.o_eoff);
        d_voff = (const unsigned long long*)(C.btab.as<char>() + bt.o_voff);
        d_fptr = (double* const*)(C.btab.as<char>() + bt.o_fptr);
    }

    RET(ensure(C.small, S_WORDS * 8));
    unsigned long long* sm = C.small.as<unsigned long long>();
    CK(cudaMemsetAsync(sm, 0, S_WORDS * 8, st));

    CK(cudaEventRecord(C.ev[1], st));
    // ---- count tet images per element ----
    RET(ensure(C.counts, (size_t)(ne + 1) * sizeof(long long)));
    RET(ensure(C.offsets, (size_t)(ne + 1) * sizeof(long long)));
    TessArgs ta = {};
    ta.m = md;
    ta.nbatch = batch ? c.nbatch : 0;
    ta.quad = m.elemtype == 27;
    for (int b = 0; batch && b < c.nbatch; ++b) ta.quad |= c.meshes[b].elemtype == 27;
    ta.meshes = d_meshes;
    ta.grids = d_grids;
    ta.eoff = d_eoff;
    ta.g = gd;
    ta.max_lvl = c.maxlvl;
    ta.refine_mode = c.refine_mode;
    ta.stretch = c.reftol;
    order_cells(c.order_cell_bits, ta.cbits);
    ta.status = (unsigned*)&sm[S_STATUS];
    ta.counters = &sm[S_TESS];
    std::vector<long long> offs_host;
    long long total = 0;
    long long klaunch = 0; // this library's own kernel launches
    {
        // counts are written as int into the first half of the buffer
        ta.e0 = 0;
        ta.e1 = ne;
        ta.count = (int*)C.counts.p;
        CK(launch_tess_count(ta, st));
        klaunch++;
        size_t tb = 0;
        const int* cin = (const int*)C.counts.p;
        long long* cout = C.offsets.as<long long>();
        CK(cudaMemsetAsync((int*)C.counts.p + ne, 0, sizeof(int), st));
        CK(cub::DeviceScan::ExclusiveScan(nullptr, tb, cin, cout, cub::Sum(), (long long)0, (int)(ne + 1), st));
        RET(ensure(C.cub_tmp, tb));
        CK(cub::DeviceScan::ExclusiveScan(C.cub_tmp.p, tb, cin, cout, cub::Sum(), (long long)0, (int)(ne + 1), st));
        CK(cudaMemcpyAsync(&total, cout + ne, sizeof(long long), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    {
        unsigned long long h[S_WORDS];
        CK(cudaMemcpy(h, sm, sizeof(h), cudaMemcpyDeviceToHost));
        RET(check_status(c, h));
    }

    // ---- chunking: images are streamed in element chunks of at most `budget` ----
    // (a capture plan keeps every image in one chunk, as the capture call has no host loop)
    long long budget = env_ll("PSIB_ITEM_BUDGET", 16ll << 20);
    if (c.capture == 1) budget = std::max(budget, total);
    std::vector<long long> cb; // element boundaries
    cb.push_back(0);
    if (total > budget) {
        offs_host.resize(ne + 1);
        CK(cudaMemcpy(offs_host.data(), C.offsets.p, (ne + 1) * sizeof(long long), cudaMemcpyDeviceToHost));
        long long e = 0;
        while (e < ne) {
            long long e1 = e;
            while (e1 < ne && offs_host[e1 + 1] - offs_host[e] <= budget) ++e1;
            if (e1 == e) e1 = e + 1; // one element larger than the budget
            cb.push_back(e1);
            e = e1;
        }
    } else {
        cb.push_back(ne);
    }
    const int nchunks = (int)cb.size() - 1;
    long long cap = 0;
    if (nchunks == 1) cap = total;
    else
        for (int k = 0; k < nchunks; ++k) cap = std::max(cap, offs_host[cb[k + 1]] - offs_host[cb[k]]);
    if (cap < 1) cap = 1;
    if (c.capture == 1) {
        // a plan: the mixed atomic walk in one chunk, with room for 25% more images in later calls
        if (!(mixed && atomic && use_bfs))
            return fail(PSIB_ERR_UNSUPPORTED, "a capture plan needs precision = mixed and deterministic = 0");
        if (nchunks != 1) return fail(PSIB_ERR_UNSUPPORTED, "a capture plan needs the images in one chunk");
        cap = total + std::max<long long>(total / 4, 4096);
    }

    RET(ensure(C.iframe, (size_t)cap * FRAME * sizeof(double)));
    RET(ensure(C.ielem, (size_t)cap * sizeof(int)));
    RET(ensure(C.ipid, (size_t)cap * 4 * sizeof(int)));
    RET(ensure(C.ikey, (size_t)cap * sizeof(uint16_t)));
    RET(ensure(C.key_sorted, (size_t)cap * sizeof(uint16_t)));
    RET(ensure(C.order_in, (size_t)cap * sizeof(int)));
    RET(ensure(C.order, (size_t)cap * sizeof(int)));
    if (central) RET(ensure(C.iscale, (size_t)cap * sizeof(double)));
    ItemArrays it;
    it.frame = C.iframe.as<double>();
    it.elem = C.ielem.as<int>();
    it.pid = C.ipid.as<int>();
    it.key = C.ikey.as<uint16_t>();
    it.grid = nullptr;
    if (batch) {
        RET(ensure(C.igrid, (size_t)cap * sizeof(uint16_t)));
        it.grid = C.igrid.as<uint16_t>();
    }
    it.cap = cap;
    ta.it = it;

    // persistent clip kernels: one resident wave, each thread with its own scratch region
    const int clip_block = 128, big_block = 64;
    const int clip_grid =
        C.num_sms * (c.adjoint ? adjoint_blocks_per_sm(false, clip_block, c.adj_coef != nullptr)
                     : central ? clip_blocks_per_sm_mixed(false, !mixed, clip_block)
                               : clip_blocks_per_sm_fp64(false, clip_block));
    const size_t main_bytes = central ? scratch_bytes_mixed(false, !mixed) : scratch_bytes_fp64(false);
    const size_t big_bytes = central ? scratch_bytes_mixed(true, !mixed) : scratch_bytes_fp64(true);
    RET(ensure(C.scratch, main_bytes * (size_t)clip_grid * clip_block));

    ClipArgs ca = {};
    ca.it = it;
    ca.order = C.order.as<int>();
    ca.g = gd;
    ca.grids = d_grids;
    ca.voff = d_voff;
    ca.mom_order = order;
    ca.status = (unsigned*)&sm[S_STATUS];
    ca.counters = &sm[S_CNT];
    ca.rec_nmom = nmom;
    ca.rec_n = &sm[S_RECN];
    ca.rec_item_base = 0;
    ca.scale = central ? C.iscale.as<double>() : nullptr;
    if (c.adjoint) {
        ca.adj_gm = c.F[0];
        ca.adj_gpos = c.gpos;
        ca.adj_npart = m.npart;
        ca.adj_gmass = c.gmass;
        ca.adj_mass_factor = m.elemtype == 4 ? 1.0 : 1.0 / 6.0;
        ca.adj_coef = c.adj_coef;
        ca.adj_gvel = c.gvel;
        ca.adj_mesh = md;
    }

    long long ntiles = 0;
    if (atomic) {
        // the per-voxel sums (only those the fields need), zeroed; the tiles' reference velocities
        int stride = 1, ox = -1, ov = -1, oxx = -1, oxv = -1, ovv = -1;
        if (flags & (F_X | F_XX | F_XV)) { ox = stride; stride += 3; }
        if (flags & (F_V | F_VV | F_XV)) { ov = stride; stride += 3; }
        if (flags & F_XX) { oxx = stride; stride += 6; }
        if (flags & F_XV) { oxv = stride; stride += 9; }
        if (flags & F_VV) { ovv = stride; stride += 6; }
        RET(ensure(C.acc_sum, (size_t)nvox * stride * sizeof(double)));
        CK(cudaMemsetAsync(C.acc_sum.p, 0, (size_t)nvox * stride * sizeof(double), st));
        // the voxels' reference points (position, velocity), claimed by their first fragments
        RET(ensure(C.acc_ref, (size_t)nvox * 2 * sizeof(unsigned long long)));
        CK(cudaMemsetAsync(C.acc_ref.p, 0, (size_t)nvox * 2 * sizeof(unsigned long long), st));
        const long long* d_toff = nullptr;
        if (batch) {
            std::vector<long long> toff(c.nbatch + 1, 0);
            for (int b = 0; b < c.nbatch; ++b) toff[b + 1] = toff[b] + acc_tiles(grid_dev(c.grids[b]));
            ntiles = toff[c.nbatch];
            RET(ensure(C.acc_toff, toff.size() * sizeof(long long)));
            CK(cudaMemcpyAsync(C.acc_toff.p, toff.data(), toff.size() * sizeof(long long), cudaMemcpyHostToDevice,
                               st));
            CK(cudaStreamSynchronize(st)); // the host table goes out of scope
            d_toff = C.acc_toff.as<long long>();
        } else {
            ntiles = acc_tiles(gd);
        }
        RET(ensure(C.acc_tsum, (size_t)ntiles * 4 * sizeof(double)));
        RET(ensure(C.acc_vref, (size_t)ntiles * 3 * sizeof(double)));
        ca.acc = AccArgs{C.acc_sum.as<double>(), stride, ox, ov, oxx, oxv, ovv, C.acc_vref.as<double>(), d_toff,
                         nullptr, C.acc_ref.as<unsigned long long>(), C.acc_ref.as<unsigned long long>() + nvox};
    }

    float ms_clip = 0.f, ms_tess = 0.f, ms_final = 0.f;
    long long corrected = 0;
    BfsSizes bsz; // the main walk's queue and pass sizes (a capture plan keeps them)
    unsigned long long clip_counts[3] = {0, 0, 0}; // fragments, fragment vertices, splits
    unsigned long long walk_bytes = 0;
    long long launches = 0;
    for (int k = 0; k < nchunks; ++k) {
        const long long e0 = cb[k], e1 = cb[k + 1];
        const long long obase = nchunks == 1 ? 0 : offs_host[e0];
        const long long nitems = nchunks == 1 ? total : offs_host[e1] - obase;
        if (nitems == 0) continue;
        if (nitems >= (1ll << 32)) return fail(PSIB_ERR_OVERFLOW, "too many tet images in one chunk");
        // ---- emit images, order them by footprint ----
        CK(cudaEventRecord(C.ev[2], st));
        ta.e0 = e0;
        ta.e1 = e1;
        ta.offset = C.offsets.as<long long>() + e0;
        ta.offset_base = obase;
        CK(launch_tess_emit(ta, st));
        CK(cudaMemsetAsync(&sm[S_NDEEP], 0, 8, st));
        k_iota<<<C.num_sms * 8, 256, 0, st>>>(C.order_in.as<int>(), nitems);
        CK(cudaGetLastError());
        k_count_deep<<<C.num_sms * 8, 256, 0, st>>>(it.key, nitems, &sm[S_NDEEP]);
        CK(cudaGetLastError());
        klaunch += 3;
        size_t tb = 0;
        CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, it.key, C.key_sorted.as<uint16_t>(), C.order_in.as<int>(),
                                           C.order.as<int>(), (int)nitems, 0, 16, st));
        RET(ensure(C.cub_tmp, tb));
        CK(cub::DeviceRadixSort::SortPairs(C.cub_tmp.p, tb, it.key, C.key_sorted.as<uint16_t>(), C.order_in.as<int>(),
                                           C.order.as<int>(), (int)nitems, 0, 16, st));
        unsigned long long hd = 0;
        CK(cudaEventRecord(C.ev[3], st));
        CK(cudaMemcpyAsync(&hd, &sm[S_NDEEP], 8, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        const long long ndeep = (long long)hd, nmain = nitems - ndeep;
        {
            float t = 0.f;
            CK(cudaEventElapsedTime(&t, C.ev[2], C.ev[3]));
            ms_tess += t;
        }

        if (c.adjoint) {
            // ---- adjoint: walk the fragments again and pull dL/dm back to the particles ----
            CK(cudaMemsetAsync(&sm[S_CNT], 0, 24, st));
            CK(cudaMemsetAsync(&sm[S_HEAD], 0, 16, st));
            CK(cudaEventRecord(C.ev[4], st));
            if (nmain > 0) {
                ca.scratch = C.scratch.p;
                ca.order_base = 0;
                ca.n = nmain;
                ca.head = &sm[S_HEAD];
                CK(launch_adjoint(ca, false, clip_grid, clip_block, st));
                launches++;
            }
            if (ndeep > 0) {
                const int big_grid = (int)std::min<long long>(
                    (long long)C.num_sms * adjoint_blocks_per_sm(true, big_block, c.adj_coef != nullptr),
                    (ndeep + big_block - 1) / big_block);
                RET(ensure(C.scratch_big, big_bytes * (size_t)big_grid * big_block));
                ca.scratch = C.scratch_big.p;
                ca.order_base = nmain;
                ca.n = ndeep;
                ca.head = &sm[S_HEAD + 1];
                CK(launch_adjoint(ca, true, big_grid, big_block, st));
                launches++;
            }
            CK(cudaEventRecord(C.ev[5], st));
            unsigned long long h[S_WORDS];
            CK(cudaMemcpyAsync(h, sm, sizeof(h), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            float t = 0.f;
            CK(cudaEventElapsedTime(&t, C.ev[4], C.ev[5]));
            ms_clip += t;
            RET(check_status(c, h));
            for (int w = 0; w < 3; ++w) clip_counts[w] += h[S_CNT + w];
            continue;
        }
        if (atomic) {
            // ---- clip, each fragment added to its voxel's sums ----
            CK(cudaMemsetAsync(&sm[S_BYTES], 0, 8, st));
            CK(cudaMemsetAsync(&sm[S_CNT], 0, 24, st));
            CK(cudaMemsetAsync(&sm[S_HEAD], 0, 16, st));
            CK(cudaEventRecord(C.ev[4], st));
            if (k == 0) {
                // the tiles' reference velocities, fixed before the first fragment is added
                CK(cudaMemsetAsync(C.acc_tsum.p, 0, (size_t)ntiles * 4 * sizeof(double), st));
                CK(launch_vref(it, nitems, gd, d_grids, ca.acc, C.acc_tsum.as<double>(), ntiles, C.num_sms, st));
                klaunch += 2;
            }
            // The deep-tree images run on a side stream beside the breadth-first walk: both add to the
            // per-voxel sums with atomics, touch disjoint images and their own scratch, and the mass
            // correction below waits for both.
            bool deep_beside = false;
            if (ndeep > 0 && nmain > 0 && use_bfs) {
                const int big_grid = (int)std::min<long long>(C.num_sms * 2, (ndeep + big_block - 1) / big_block);
                RET(ensure(C.scratch_big, big_bytes * (size_t)big_grid * big_block));
                ClipArgs cd = ca;
                cd.scratch = C.scratch_big.p;
                cd.order_base = nmain;
                cd.n = ndeep;
                cd.head = &sm[S_HEAD + 1];
                CK(cudaEventRecord(C.fork, st));
                CK(cudaStreamWaitEvent(C.side, C.fork, 0));
                CK(launch_clip_mixed(cd, true, !mixed, big_grid, big_block, C.side));
                CK(cudaEventRecord(C.join, C.side));
                launches++;
                deep_beside = true;
            }
            if (nmain > 0 && use_bfs) {
                ca.scratch = C.scratch.p;
                RET(bfs_clip(C, ca, nmain, nitems, sm, clip_grid, clip_block, c.queue_voxels, batch, st, launches,
                             klaunch, C.key_sorted.as<uint16_t>(), &bsz));
            } else if (nmain > 0) {
                ca.scratch = C.scratch.p;
                ca.order_base = 0;
                ca.n = nmain;
                ca.head = &sm[S_HEAD];
                CK(launch_clip_mixed(ca, false, !mixed, clip_grid, clip_block, st));
                launches++;
            }
            if (deep_beside) {
                CK(cudaStreamWaitEvent(st, C.join, 0));
            } else if (ndeep > 0) {
                const int big_grid = (int)std::min<long long>(C.num_sms * 2, (ndeep + big_block - 1) / big_block);
                RET(ensure(C.scratch_big, big_bytes * (size_t)big_grid * big_block));
                ca.scratch = C.scratch_big.p;
                ca.order_base = nmain;
                ca.n = ndeep;
                ca.head = &sm[S_HEAD + 1];
                CK(launch_clip_mixed(ca, true, !mixed, big_grid, big_block, st));
                launches++;
            }
            if (nmain > 0 && use_bfs) {
                // every image's scale is set now (the deep-tree kernel sets its own to 1)
                long long ncorr = 0;
                RET(correct_masses(C, ca, nitems, sm, clip_grid, clip_block, c.queue_voxels, st, launches, klaunch,
                                   ncorr));
                corrected += ncorr;
            }
            CK(cudaEventRecord(C.ev[5], st));
            unsigned long long h[S_WORDS];
            CK(cudaMemcpyAsync(h, sm, sizeof(h), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            float t = 0.f;
            CK(cudaEventElapsedTime(&t, C.ev[4], C.ev[5]));
            ms_clip += t;
            RET(check_status(c, h));
            for (int w = 0; w < 3; ++w) clip_counts[w] += h[S_CNT + w];
            walk_bytes += h[S_BYTES];
            continue;
        }
        // ---- clip to fragment records; grow the record buffer and redo if it overflowed ----
        int ibits = 1, vbits = 1;
        while ((1ll << ibits) < nitems) ++ibits;
        while ((1ll << vbits) < nvox) ++vbits;
        if (ibits + vbits > 64) return fail(PSIB_ERR_OVERFLOW, "grid and chunk too large for a 64-bit record key");
        ca.rec_ibits = ibits;
        for (int attempt = 0;; ++attempt) {
            const unsigned long long want = (unsigned long long)std::max<long long>(nitems * 20, 1 << 16);
            const unsigned long long have = std::max<unsigned long long>(C.rkey.n / 8, want);
            RET(ensure(C.rkey, have * 8));
            RET(ensure(C.rmom, have * 8 * nmom));
            ca.rec_key = C.rkey.as<unsigned long long>();
            ca.rec_mom = C.rmom.as<double>();
            ca.rec_cap = std::min<unsigned long long>(C.rkey.n / 8, C.rmom.n / (8 * nmom));
            CK(cudaMemsetAsync(&sm[S_RECN], 0, 8, st));
            CK(cudaMemsetAsync(&sm[S_BYTES], 0, 8, st));
            CK(cudaMemsetAsync(&sm[S_CNT], 0, 24, st)); // this attempt's counters
            CK(cudaMemsetAsync(&sm[S_HEAD], 0, 16, st));
            CK(cudaEventRecord(C.ev[4], st));
            // Beside the FP64 walk, the deep-tree images run on the side stream: both reserve record
            // slots with atomics (the sort puts them in order) and use their own scratch and queue heads.
            bool deep_beside = false;
            if (ndeep > 0 && nmain > 0 && use_bfs64) {
                const int big_grid = (int)std::min<long long>(C.num_sms * 2, (ndeep + big_block - 1) / big_block);
                RET(ensure(C.scratch_big, big_bytes * (size_t)big_grid * big_block));
                ClipArgs cd = ca;
                cd.scratch = C.scratch_big.p;
                cd.order_base = nmain;
                cd.n = ndeep;
                cd.head = &sm[S_HEAD + 1];
                CK(cudaEventRecord(C.fork, st));
                CK(cudaStreamWaitEvent(C.side, C.fork, 0));
                CK(launch_clip_fp64(cd, true, big_grid, big_block, C.side));
                CK(cudaEventRecord(C.join, C.side));
                launches++;
                deep_beside = true;
            }
            if (nmain > 0 && (use_bfs || use_bfs64)) {
                ca.scratch = C.scratch.p;
                RET(bfs_clip(C, ca, nmain, nitems, sm, clip_grid, clip_block, c.queue_voxels, batch, st, launches,
                             klaunch, C.key_sorted.as<uint16_t>(), nullptr, use_bfs64));
            } else if (nmain > 0) {
                ca.scratch = C.scratch.p;
                ca.order_base = 0;
                ca.n = nmain;
                ca.head = &sm[S_HEAD];
                if (central) CK(launch_clip_mixed(ca, false, !mixed, clip_grid, clip_block, st));
                else CK(launch_clip_fp64(ca, false, clip_grid, clip_block, st));
                launches++;
            }
            if (deep_beside) {
                CK(cudaStreamWaitEvent(st, C.join, 0));
            } else if (ndeep > 0) {
                const int big_grid = (int)std::min<long long>(C.num_sms * 2, (ndeep + big_block - 1) / big_block);
                RET(ensure(C.scratch_big, big_bytes * (size_t)big_grid * big_block));
                ca.scratch = C.scratch_big.p;
                ca.order_base = nmain;
                ca.n = ndeep;
                ca.head = &sm[S_HEAD + 1];
                if (central) CK(launch_clip_mixed(ca, true, !mixed, big_grid, big_block, st));
                else CK(launch_clip_fp64(ca, true, big_grid, big_block, st));
                launches++;
            }
            CK(cudaEventRecord(C.ev[5], st));
            unsigned long long h[S_WORDS];
            CK(cudaMemcpyAsync(h, sm, sizeof(h), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            {
                float t = 0.f;
                CK(cudaEventElapsedTime(&t, C.ev[4], C.ev[5]));
                ms_clip += t;
            }
            const unsigned long long nrec = h[S_RECN];
            if (nrec > ca.rec_cap && attempt == 0) {
                // the buffer was too small: grow to the exact need and redo the chunk
                RET(ensure(C.rkey, nrec * 8));
                RET(ensure(C.rmom, nrec * 8 * nmom));
                unsigned clr = 0;
                CK(cudaMemcpy(&sm[S_STATUS], &clr, sizeof(clr), cudaMemcpyHostToDevice));
                continue;
            }
            RET(check_status(c, h));
            for (int w = 0; w < 3; ++w) clip_counts[w] += h[S_CNT + w];
            walk_bytes += h[S_BYTES];
            if (nrec >= (1ull << 32)) return fail(PSIB_ERR_OVERFLOW, "too many fragments in one chunk");
            if (nrec == 0) break;
            // ---- sort records by (voxel, image), gather them in that order, apply each voxel's run ----
            CK(cudaEventRecord(C.ev[6], st));
            RET(ensure(C.rkey_sorted, nrec * 8));
            RET(ensure(C.rperm_in, nrec * 4));
            RET(ensure(C.rperm, nrec * 4));
            RET(ensure(C.rvox, nrec * 4));
            RET(ensure(C.ritem, nrec * 4));
            if (!central) RET(ensure(C.rmom_sorted, nrec * 8 * nmom));
            const long long maxruns = std::min<long long>((long long)nrec, nvox);
            RET(ensure(C.run_vox, (size_t)maxruns * 4));
            RET(ensure(C.run_cnt, (size_t)maxruns * 4 + 8));
            RET(ensure(C.run_off, (size_t)maxruns * 8));
            k_iota<<<C.num_sms * 8, 256, 0, st>>>(C.rperm_in.as<unsigned>(), (long long)nrec);
            CK(cudaGetLastError());
            tb = 0;
            CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, C.rkey.as<unsigned long long>(),
                                               C.rkey_sorted.as<unsigned long long>(), C.rperm_in.as<unsigned>(),
                                               C.rperm.as<unsigned>(), (int)nrec, 0, ibits + vbits, st));
            RET(ensure(C.cub_tmp, tb));
            CK(cub::DeviceRadixSort::SortPairs(C.cub_tmp.p, tb, C.rkey.as<unsigned long long>(),
                                               C.rkey_sorted.as<unsigned long long>(), C.rperm_in.as<unsigned>(),
                                               C.rperm.as<unsigned>(), (int)nrec, 0, ibits + vbits, st));
            GatherArgs ga = {};
            ga.key = C.rkey_sorted.as<unsigned long long>();
            ga.perm = C.rperm.as<unsigned>();
            ga.mom = C.rmom.as<double>();
            ga.nrec = (long long)nrec;
            ga.nmom = nmom;
            ga.ibits = ibits;
            ga.vox = C.rvox.as<unsigned>();
            ga.item = C.ritem.as<unsigned>();
            ga.mom_sorted = central ? nullptr : C.rmom_sorted.as<double>();
            CK(launch_gather_records(ga, st));
            // voxel runs: (voxel, count) pairs, then their offsets
            int* d_nruns = (int*)(C.run_cnt.as<char>() + (size_t)maxruns * 4);
            tb = 0;
            CK(cub::DeviceRunLengthEncode::Encode(nullptr, tb, C.rvox.as<unsigned>(), C.run_vox.as<unsigned>(),
                                                  C.run_cnt.as<int>(), d_nruns, (int)nrec, st));
            RET(ensure(C.cub_tmp, tb));
            CK(cub::DeviceRunLengthEncode::Encode(C.cub_tmp.p, tb, C.rvox.as<unsigned>(), C.run_vox.as<unsigned>(),
                                                  C.run_cnt.as<int>(), d_nruns, (int)nrec, st));
            int nruns = 0;
            CK(cudaMemcpyAsync(&nruns, d_nruns, sizeof(int), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            tb = 0;
            CK(cub::DeviceScan::ExclusiveScan(nullptr, tb, C.run_cnt.as<int>(), C.run_off.as<long long>(), cub::Sum(),
                                              (long long)0, nruns, st));
            RET(ensure(C.cub_tmp, tb));
            CK(cub::DeviceScan::ExclusiveScan(C.cub_tmp.p, tb, C.run_cnt.as<int>(), C.run_off.as<long long>(),
                                              cub::Sum(), (long long)0, nruns, st));
            ApplyArgs aa = {};
            aa.run_vox = C.run_vox.as<unsigned>();
            aa.run_cnt = C.run_cnt.as<int>();
            aa.run_off = C.run_off.as<long long>();
            aa.nruns = nruns;
            aa.item = C.ritem.as<unsigned>();
            aa.mom = central ? C.rmom.as<double>() : C.rmom_sorted.as<double>();
            aa.perm = C.rperm.as<unsigned>();
            aa.nmom = nmom;
            aa.central = central;
            aa.scale = ca.scale;
            aa.it = it;
            aa.item_base = 0;
            aa.M = c.F[0]; aa.X = c.F[1]; aa.V = c.F[2]; aa.XX = c.F[3]; aa.XV = c.F[4]; aa.VV = c.F[5];
            aa.nbatch = batch ? c.nbatch : 0;
            aa.voff = d_voff;
            aa.fptr = d_fptr;
            // host-memory calls copy the fields in beside the first stages; only this one needs them
            if (c.fields_ready) CK(cudaStreamWaitEvent(st, c.fields_ready, 0));
            if (c.host_fields && k == nchunks - 1 && !batch && nruns >= 4 * NOUT) {
                // The last chunk: apply the runs in NOUT slabs of voxels (runs are sorted by
                // voxel) and copy each slab of every field to the host on the copy stream
                // while the next slab is applied.
                long long rb[NOUT + 1];
                unsigned vb[NOUT + 1];
                for (int p = 0; p <= NOUT; ++p) rb[p] = (long long)nruns * p / NOUT;
                vb[0] = 0;
                vb[NOUT] = (unsigned)nvox;
                for (int p = 1; p < NOUT; ++p)
                    CK(cudaMemcpyAsync(&vb[p], C.run_vox.as<unsigned>() + rb[p], sizeof(unsigned),
                                       cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
                static const int comps[6] = {1, 3, 3, 9, 9, 9};
                for (int p = 0; p < NOUT; ++p) {
                    ApplyArgs ap = aa;
                    ap.run_vox = aa.run_vox + rb[p];
                    ap.run_cnt = aa.run_cnt + rb[p];
                    ap.run_off = aa.run_off + rb[p];
                    ap.nruns = rb[p + 1] - rb[p];
                    CK(launch_apply_records(ap, st));
                    CK(cudaEventRecord(C.ev_out[p], st));
                    CK(cudaStreamWaitEvent(C.copy, C.ev_out[p], 0));
                    for (int f = 0; f < 6; ++f) {
                        if (!c.F[f]) continue;
                        const size_t o = (size_t)vb[p] * comps[f] * sizeof(double);
                        const size_t n = (size_t)(vb[p + 1] - vb[p]) * comps[f] * sizeof(double);
                        CK(cudaMemcpyAsync((char*)c.host_fields[f] + o, (const char*)c.F[f] + o, n,
                                           cudaMemcpyDeviceToHost, C.copy));
                    }
                }
                c.copied_out = true;
                klaunch += NOUT - 1;
            } else {
                CK(launch_apply_records(aa, st));
            }
            klaunch += 3; // iota, gather, apply
            CK(cudaEventRecord(C.ev[7], st));
            CK(cudaEventSynchronize(C.ev[7]));
            float t = 0.f;
            CK(cudaEventElapsedTime(&t, C.ev[6], C.ev[7]));
            ms_final += t;
            break;
        }
    }
    if (atomic) {
        // ---- merge every voxel's sums into its fields; host calls copy each slab back beside the next ----
        CK(cudaEventRecord(C.ev[6], st));
        FinalArgs fa = {};
        fa.ap.M = c.F[0]; fa.ap.X = c.F[1]; fa.ap.V = c.F[2]; fa.ap.XX = c.F[3]; fa.ap.XV = c.F[4]; fa.ap.VV = c.F[5];
        fa.ap.nbatch = batch ? c.nbatch : 0;
        fa.ap.voff = d_voff;
        fa.ap.fptr = d_fptr;
        fa.acc = ca.acc;
        fa.g = gd;
        fa.grids = d_grids;
        if (c.fields_ready) CK(cudaStreamWaitEvent(st, c.fields_ready, 0));
        if (c.host_fields && !batch && nvox >= 4 * NOUT) {
            static const int comps[6] = {1, 3, 3, 9, 9, 9};
            for (int p = 0; p < NOUT; ++p) {
                fa.v0 = nvox * p / NOUT;
                fa.v1 = nvox * (p + 1) / NOUT;
                CK(launch_acc_finalize(fa, C.num_sms, st));
                CK(cudaEventRecord(C.ev_out[p], st));
                CK(cudaStreamWaitEvent(C.copy, C.ev_out[p], 0));
                for (int f = 0; f < 6; ++f) {
                    if (!c.F[f]) continue;
                    const size_t o = (size_t)fa.v0 * comps[f] * sizeof(double);
                    const size_t n = (size_t)(fa.v1 - fa.v0) * comps[f] * sizeof(double);
                    CK(cudaMemcpyAsync((char*)c.host_fields[f] + o, (const char*)c.F[f] + o, n,
                                       cudaMemcpyDeviceToHost, C.copy));
                }
            }
            c.copied_out = true;
            klaunch += NOUT;
        } else {
            fa.v0 = 0;
            fa.v1 = nvox;
            CK(launch_acc_finalize(fa, C.num_sms, st));
            klaunch++;
        }
        CK(cudaEventRecord(C.ev[7], st));
        CK(cudaEventSynchronize(C.ev[7]));
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, C.ev[6], C.ev[7]));
        ms_final += t;
    }
    unsigned long long h[S_WORDS];
    CK(cudaMemcpyAsync(h, sm, sizeof(h), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    RET(check_status(c, h));
    if (c.capture == 1) {
        // the plan of later capture calls: every buffer they use, sized now
        Ctx::Plan& P = C.plan;
        P = Ctx::Plan{};
        P.nelem = ne;
        P.nbatch = batch ? c.nbatch : 0;
        P.nvox = nvox;
        P.cap_items = cap;
        P.ntiles = ntiles;
        P.stride = ca.acc.stride;
        P.flags = flags;
        P.precision = c.precision;
        P.tiles = std::max<long long>(bsz.tiles, 1);
        P.qcap = P.tiles * 32; // the queues as allocated: a capture call's passes must fit them
        P.max_passes = (int)std::max<long long>(bsz.npass, 1) + 2;
        P.btab_bytes = batch ? C.btab_host_n : 0;
        RET(ensure(C.passes, (size_t)(P.max_passes + 1) * sizeof(long long)));
        RET(ensure(C.fix_list, (size_t)cap * sizeof(int)));
        RET(ensure(C.fix_keys, (size_t)cap * sizeof(uint16_t)));
        RET(ensure(C.ifactor, (size_t)cap * sizeof(double)));
        RET(ensure(C.vsum, (size_t)cap * sizeof(double)));
        RET(ensure(C.dfs_list, (size_t)cap * sizeof(int)));
        const int big_grid = C.num_sms * 2;
        RET(ensure(C.scratch_big, big_bytes * (size_t)big_grid * big_block));
        size_t tb = 0, t2 = 0;
        CK(cub::DeviceScan::ExclusiveScan(nullptr, tb, (const int*)C.counts.p, C.offsets.as<long long>(), cub::Sum(),
                                          (long long)0, (int)(ne + 1), st));
        CK(cub::DeviceRadixSort::SortPairs(nullptr, t2, it.key, C.key_sorted.as<uint16_t>(), C.order_in.as<int>(),
                                           C.order.as<int>(), (int)cap, 0, 16, st));
        RET(ensure(C.cub_tmp, std::max(tb, t2)));
        P.valid = true;
    }
    if (c.stats) {
        psib_stats& s = *c.stats;
        s.corrected_items = corrected;
        s.accumulation = atomic ? 1 : 0;
        s.elements_kept = (long long)h[S_TESS];
        s.tets = (long long)h[S_TESS + 1];
        s.tet_images = total;
        s.fragments = (long long)clip_counts[0];
        s.frag_verts = (long long)clip_counts[1];
        s.splits = (long long)clip_counts[2];
        s.passes = 1;
        s.chunks = nchunks;
        s.ms_clip = ms_clip;
        s.ms_tess = ms_tess;
        s.ms_final = ms_final;
        s.clip_launches = launches;
        s.kernel_launches = klaunch + launches;
        s.walk_bytes = (long long)walk_bytes;
    }
    (void)nvox;
    return PSIB_OK;
}

// ---- capture mode: a call without host synchronisation or allocation ----

// The mixed atomic deposit of run_device with every count kept on the device and every buffer
// taken from the plan call before it (options.capture = 1), so that the caller can record the
// call in a CUDA graph.  The item buffer has the plan's fixed size: its unused entries get
// KEY_PAD and sort past the images; the main and deep images are counted on the device; a
// one-thread kernel lays out the walk's passes (k_plan_passes) and the plan's number of passes is
// launched, those beyond the need walking nothing; the deep-tree kernel and the mass-correction
// pass read their sizes from the device.  Failures stay in the device status word
// (psib_capture_status).
int run_capture(Call& c)
{
    Ctx& C = *c.C;
    const Ctx::Plan& P = C.plan;
    const psib_grid& g = *c.grid;
    const psib_mesh& m = *c.mesh;
    cudaStream_t st = c.st;
    const bool batch = c.nbatch > 0;
    long long nvox = (long long)g.n[0] * g.n[1] * g.n[2];
    long long ne = m.nelem;
    std::vector<long long> eoff{0};
    std::vector<unsigned long long> voff{0};
    if (batch) {
        for (int b = 0; b < c.nbatch; ++b) {
            const psib_grid& gb = c.grids[b];
            eoff.push_back(eoff.back() + c.meshes[b].nelem);
            voff.push_back(voff.back() + (unsigned long long)gb.n[0] * gb.n[1] * gb.n[2]);
        }
        nvox = (long long)voff.back();
        ne = eoff.back();
    }
    unsigned flags = 0;
    if (c.F[1]) flags |= F_X;
    if (c.F[2]) flags |= F_V;
    if (c.F[3]) flags |= F_XX;
    if (c.F[4]) flags |= F_XV;
    if (c.F[5]) flags |= F_VV;
    if (!P.valid || P.nelem != ne || P.nvox != nvox || P.nbatch != (batch ? c.nbatch : 0) || P.flags != flags ||
        P.precision != c.precision)
        return fail(PSIB_ERR_ARG, "a capture call needs a plan call (options.capture = 1) with the same grids, meshes "
                                  "and fields before it");
    if (c.precision != PSIB_MIXED || c.deterministic || c.adjoint || c.mode != PSIB_MODE_DENSITY)
        return fail(PSIB_ERR_UNSUPPORTED, "the capture mode runs the mixed atomic deposit");
    const int order = (flags & (F_XX | F_XV | F_VV)) ? 2 : (flags & (F_X | F_V)) ? 1 : 0;
    const long long cap = P.cap_items;
    const GridDev gd = grid_dev(g);
    const MeshDev md = mesh_dev(m, g, c.pos, c.vel, c.mass, c.conn, c.reftol, c.refine_cell);
    const MeshDev* d_meshes = nullptr;
    const GridDev* d_grids = nullptr;
    const long long* d_eoff = nullptr;
    const unsigned long long* d_voff = nullptr;
    double* const* d_fptr = nullptr;
    if (batch) {
        BatchTables bt;
        RET(batch_tables(c, eoff, voff, bt));
        if (bt.h.size() > C.btab_host_n || bt.h.size() > C.btab.n)
            return fail(PSIB_ERR_ARG, "the batch tables outgrew the plan");
        memcpy(C.btab_host, bt.h.data(), bt.h.size()); // page-locked: read when the copy runs
        CK(cudaMemcpyAsync(C.btab.p, C.btab_host, bt.h.size(), cudaMemcpyHostToDevice, st));
        d_meshes = (const MeshDev*)(C.btab.as<char>() + bt.o_mesh);
        d_grids = (const GridDev*)(C.btab.as<char>() + bt.o_grid);
        d_eoff = (const long long*)(C.btab.as<char>() + bt.o_eoff);
        d_voff = (const unsigned long long*)(C.btab.as<char>() + bt.o_voff);
        d_fptr = (double* const*)(C.btab.as<char>() + bt.o_fptr);
    }
    unsigned long long* sm = C.small.as<unsigned long long>();
    unsigned* status = (unsigned*)&sm[S_STATUS];
    CK(cudaMemsetAsync(&sm[1], 0, (S_WORDS - 1) * 8, st)); // the status word keeps earlier failures

    // images: count, scan, emit into the fixed buffer, pad, order
    TessArgs ta = {};
    ta.m = md;
    ta.nbatch = batch ? c.nbatch : 0;
    ta.quad = m.elemtype == 27;
    for (int b = 0; batch && b < c.nbatch; ++b) ta.quad |= c.meshes[b].elemtype == 27;
    ta.meshes = d_meshes;
    ta.grids = d_grids;
    ta.eoff = d_eoff;
    ta.g = gd;
    ta.max_lvl = c.maxlvl;
    ta.refine_mode = c.refine_mode;
    ta.stretch = c.reftol;
    order_cells(c.order_cell_bits, ta.cbits);
    ta.status = status;
    ta.counters = &sm[S_TESS];
    ta.e0 = 0;
    ta.e1 = ne;
    ta.count = (int*)C.counts.p;
    CK(launch_tess_count(ta, st));
    CK(cudaMemsetAsync((int*)C.counts.p + ne, 0, sizeof(int), st));
    size_t tb = 0;
    CK(cub::DeviceScan::ExclusiveScan(nullptr, tb, (const int*)C.counts.p, C.offsets.as<long long>(), cub::Sum(),
                                      (long long)0, (int)(ne + 1), st));
    if (tb > C.cub_tmp.n) return fail(PSIB_ERR_ARG, "scan scratch outgrew the plan");
    CK(cub::DeviceScan::ExclusiveScan(C.cub_tmp.p, tb, (const int*)C.counts.p, C.offsets.as<long long>(),
                                      cub::Sum(), (long long)0, (int)(ne + 1), st));
    const long long* total_dev = C.offsets.as<long long>() + ne;
    ItemArrays it;
    it.frame = C.iframe.as<double>();
    it.elem = C.ielem.as<int>();
    it.pid = C.ipid.as<int>();
    it.key = C.ikey.as<uint16_t>();
    it.grid = batch ? C.igrid.as<uint16_t>() : nullptr;
    it.cap = cap;
    ta.it = it;
    ta.offset = C.offsets.as<long long>();
    ta.offset_base = 0;
    CK(launch_tess_emit(ta, st));
    k_pad_keys<<<C.num_sms * 8, 256, 0, st>>>(it.key, total_dev, cap);
    k_iota<<<C.num_sms * 8, 256, 0, st>>>(C.order_in.as<int>(), cap);
    CK(cudaGetLastError());
    tb = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, it.key, C.key_sorted.as<uint16_t>(), C.order_in.as<int>(),
                                       C.order.as<int>(), (int)cap, 0, 16, st));
    if (tb > C.cub_tmp.n) return fail(PSIB_ERR_ARG, "sort scratch outgrew the plan");
    CK(cub::DeviceRadixSort::SortPairs(C.cub_tmp.p, tb, it.key, C.key_sorted.as<uint16_t>(), C.order_in.as<int>(),
                                       C.order.as<int>(), (int)cap, 0, 16, st));
    k_key_classes<<<C.num_sms * 8, 256, 0, st>>>(C.key_sorted.as<uint16_t>(), cap, &sm[S_NMAIN], &sm[S_NDEEP]);
    CK(cudaGetLastError());

    // the per-voxel sums and the tiles' reference velocities
    CK(cudaMemsetAsync(C.acc_sum.p, 0, (size_t)nvox * P.stride * sizeof(double), st));
    CK(cudaMemsetAsync(C.acc_ref.p, 0, (size_t)nvox * 2 * sizeof(unsigned long long), st));
    ClipArgs ca = {};
    ca.it = it;
    ca.order = C.order.as<int>();
    ca.g = gd;
    ca.grids = d_grids;
    ca.voff = d_voff;
    ca.mom_order = order;
    ca.status = status;
    ca.counters = &sm[S_CNT];
    ca.rec_nmom = order == 2 ? 10 : order == 1 ? 4 : 1;
    ca.rec_n = &sm[S_RECN];
    ca.scale = C.iscale.as<double>();
    {
        int stride = 1, ox = -1, ov = -1, oxx = -1, oxv = -1, ovv = -1;
        if (flags & (F_X | F_XX | F_XV)) { ox = stride; stride += 3; }
        if (flags & (F_V | F_VV | F_XV)) { ov = stride; stride += 3; }
        if (flags & F_XX) { oxx = stride; stride += 6; }
        if (flags & F_XV) { oxv = stride; stride += 9; }
        if (flags & F_VV) { ovv = stride; stride += 6; }
        ca.acc = AccArgs{C.acc_sum.as<double>(), stride, ox, ov, oxx, oxv, ovv, C.acc_vref.as<double>(),
                         batch ? C.acc_toff.as<long long>() : nullptr, nullptr, C.acc_ref.as<unsigned long long>(),
                         C.acc_ref.as<unsigned long long>() + nvox};
    }
    CK(cudaMemsetAsync(C.acc_tsum.p, 0, (size_t)P.ntiles * 4 * sizeof(double), st));
    CK(launch_vref(it, cap, gd, d_grids, ca.acc, C.acc_tsum.as<double>(), P.ntiles, C.num_sms, st, total_dev));

    // the breadth-first walk of the main images, its passes planned on the device
    PolyQueue Q[3];
    const size_t tiles = (size_t)P.tiles;
    for (int i = 0; i < 3; ++i)
        Q[i] = PolyQueue{C.qx[i].as<float>(), C.qnb[i].as<uint32_t>(), C.qnv[i].as<uint8_t>(),
                         C.qwin[i].as<uint8_t>(), C.qbox[i].as<uint32_t>(), C.qitem[i].as<uint32_t>(), nullptr,
                         (unsigned long long)tiles * 32};
    unsigned long long* cq = C.bfs_cnt.as<unsigned long long>();
    BfsArgs ba = {};
    ba.c = ca;
    ba.dfs_list = C.dfs_list.as<int>();
    ba.dfs_count = &sm[S_DFS];
    ba.bytes = &sm[S_BYTES];
    ba.window_bfs = 1;
    ba.level_blocks = (int)env_ll("PSIB_LEVEL_BLOCKS", 0); // as bfs_clip
    ba.leaf_split = (int)env_ll("PSIB_LEAF_SPLIT", 7);
    ba.level_split = (int)env_ll("PSIB_LEVEL_SPLIT", 0);
    ba.vsum = C.vsum.as<double>();
    ba.passes = C.passes.as<long long>();
    ba.pass_idx = &sm[S_PASS];
    CK(cudaMemsetAsync(C.hist.p, 0, (65536 >> KEY_CELL_BITS) * sizeof(unsigned), st));
    k_key_hist_dev<<<C.num_sms * 4, 256, 0, st>>>(C.key_sorted.as<uint16_t>(), &sm[S_NMAIN], C.hist.as<unsigned>());
    k_plan_passes<<<1, 1, 0, st>>>(C.hist.as<unsigned>(), P.qcap, C.passes.as<long long>(), P.max_passes,
                                   &sm[S_NMAIN], status);
    CK(cudaGetLastError());
    for (int p = 0; p < P.max_passes; ++p) CK(bfs_pass(ba, Q, cq, C.num_sms, st));
    CK(launch_bfs_finalize(ba, cap, C.num_sms, st));

    // the deep-tree images, their number and first position read on the device
    {
        const int big_block = 64, big_grid = C.num_sms * 2;
        ClipArgs cd = ca;
        cd.scratch = C.scratch_big.p;
        cd.n_dev = &sm[S_NDEEP];
        cd.base_dev = &sm[S_NMAIN];
        cd.n = 0;
        cd.head = &sm[S_HEAD + 1];
        CK(launch_clip_mixed(cd, true, false, big_grid, big_block, st));
    }

    // images whose FP32 walk missed their exact volume: walked again with their mass factor
    CK(launch_correction_select(it, ca.scale, cap, 1e-14, C.fix_list.as<int>(), C.fix_keys.as<uint16_t>(),
                                C.ifactor.as<double>(), &sm[S_FIX], C.num_sms, st, total_dev));
    k_plan_list<<<1, 256, 0, st>>>(C.fix_keys.as<uint16_t>(), &sm[S_FIX], P.qcap, C.passes.as<long long>(),
                                   P.max_passes, status);
    CK(cudaGetLastError());
    {
        BfsArgs bf = ba;
        bf.c.order = C.fix_list.as<int>();
        bf.c.acc.factor = C.ifactor.as<double>();
        CK(cudaMemsetAsync(&sm[S_PASS], 0, 8, st));
        CK(bfs_pass(bf, Q, cq, C.num_sms, st));
    }

    // every voxel's sums into its fields
    FinalArgs fa = {};
    fa.ap.M = c.F[0]; fa.ap.X = c.F[1]; fa.ap.V = c.F[2]; fa.ap.XX = c.F[3]; fa.ap.XV = c.F[4]; fa.ap.VV = c.F[5];
    fa.ap.nbatch = batch ? c.nbatch : 0;
    fa.ap.voff = d_voff;
    fa.ap.fptr = d_fptr;
    fa.acc = ca.acc;
    fa.g = gd;
    fa.grids = d_grids;
    fa.v0 = 0;
    fa.v1 = nvox;
    CK(launch_acc_finalize(fa, C.num_sms, st));
    return PSIB_OK;
}

} // namespace

int psib::report_error(int code, const char* msg) { return fail(code, "%s", msg); }

extern "C" {

const char* psib_last_error(void) { return g_err.c_str(); }

int psib_abi_version(void) { return PSIB_ABI_VERSION; }

int psib_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

void* psib_host_alloc(unsigned long long bytes)
{
    void* p = nullptr;
    if (psib_device_count() <= 0) return nullptr;
    if (cudaHostAlloc(&p, bytes ? bytes : 16, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

void psib_host_free(void* p)
{
    if (p) cudaFreeHost(p);
}

int psib_release_device_memory(void)
{
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_mu);
    if (dev >= 0 && dev < 64 && g_ctx[dev]) {
        CK(cudaDeviceSynchronize());
        if (g_ctx[dev]->pass_exec) cudaGraphExecDestroy(g_ctx[dev]->pass_exec); // it refers to the buffers
        g_ctx[dev]->pass_exec = nullptr;
        for (DevBuf* b : g_ctx[dev]->all()) {
            if (b->p) cudaFree(b->p);
            b->p = nullptr;
            b->n = 0;
        }
    }
    return PSIB_OK;
}

int psib_voxels(const psib_grid* grid, const psib_mesh* mesh, int mode, double refine_tolerance, int refine_max_lvl,
                const psib_options* opt)
{
    g_err.clear();
    psib_options o = {};
    o.precision = PSIB_FP64;
    o.memory = PSIB_HOST;
    o.device = -1;
    if (opt) o = *opt;
    RET(validate(grid, mesh, mode, &o));
    if (psib_device_count() <= 0) return fail(PSIB_ERR_NODEVICE, "no CUDA device is visible");
    int dev = o.device;
    if (o.memory == PSIB_DEVICE || dev < 0) CK(cudaGetDevice(&dev));
    CK(cudaSetDevice(dev));
    Ctx* C = nullptr;
    RET(get_ctx(dev, &C));

    Call c = {};
    c.grid = grid;
    c.mesh = mesh;
    c.mode = mode;
    c.reftol = refine_tolerance;
    c.maxlvl = refine_max_lvl > 6 ? 6 : (refine_max_lvl < 0 ? 0 : refine_max_lvl);
    c.precision = o.precision;
    c.deterministic = o.deterministic;
    c.refine_mode = o.refine_mode;
    c.queue_voxels = o.queue_voxels;
    c.capture = o.capture;
    c.order_cell_bits = o.order_cell_bits;
    if (o.capture && o.memory != PSIB_DEVICE) return fail(PSIB_ERR_ARG, "the capture mode takes device memory");
    if (o.refine_mode == PSIB_REFINE_STRETCH) {
        const bool given = o.refine_cell[0] > 0.0 && o.refine_cell[1] > 0.0 && o.refine_cell[2] > 0.0;
        for (int i = 0; i < 3; ++i) {
            if (given) c.refine_cell[i] = o.refine_cell[i];
            else if (mesh->periodic && mesh->block_dims[i] > 0)
                c.refine_cell[i] = (mesh->box[1][i] - mesh->box[0][i]) / mesh->block_dims[i];
            else return fail(PSIB_ERR_ARG, "the stretch criterion needs refine_cell or a periodic block mesh");
        }
        if (!(refine_tolerance > 0.0)) return fail(PSIB_ERR_ARG, "the stretch threshold must be positive");
    }
    c.C = C;
    c.stats = o.stats;
    if (o.stats) *o.stats = psib_stats{};

    const long long nvox = (long long)grid->n[0] * grid->n[1] * grid->n[2];
    static const int comps[6] = {1, 3, 3, 9, 9, 9};
    if (o.memory == PSIB_DEVICE) {
        RET(enter_own_stream(*C, (cudaStream_t)o.stream));
        c.st = C->own;
        for (int f = 0; f < 6; ++f) c.F[f] = grid->fields[f];
        c.pos = mesh->pos;
        c.vel = mesh->vel;
        c.mass = mesh->mass;
        c.conn = mesh->connectivity;
        if (o.capture == 2) {
            c.stats = nullptr;
            const int r = run_capture(c);
            RET(leave_own_stream(*C, (cudaStream_t)o.stream));
            return r;
        }
        CK(cudaEventRecord(C->ev[0], c.st));
        const int r = run_device(c);
        RET(leave_own_stream(*C, (cudaStream_t)o.stream));
        RET(r);
        if (o.stats) {
            CK(cudaEventRecord(C->ev[7], c.st));
            CK(cudaEventSynchronize(C->ev[7]));
            CK(cudaEventElapsedTime(&o.stats->ms_total, C->ev[0], C->ev[7]));
        }
        return PSIB_OK;
    }
    // host memory: copy in, run, copy out
    cudaStream_t st = C->own;
    c.st = st;
    CK(cudaEventRecord(C->ev[0], st));
    if (mesh->nelem > 0) RET(copy_mesh_in(c, *C, *mesh, st));
    // the grid fields travel on a second stream while the mesh is tessellated and clipped;
    // the field update waits for them (the previous call ended with a synchronize, so the
    // device copies are free)
    for (int f = 0; f < 6; ++f) {
        if (!grid->fields[f]) continue;
        const size_t b = (size_t)nvox * comps[f] * sizeof(double);
        RET(ensure(C->hfield[f], b));
        CK(cudaMemcpyAsync(C->hfield[f].p, grid->fields[f], b, cudaMemcpyHostToDevice, C->copy));
        c.F[f] = C->hfield[f].as<double>();
    }
    CK(cudaEventRecord(C->fields_in, C->copy));
    c.fields_ready = C->fields_in;
    c.host_fields = grid->fields;
    if (mesh->nelem > 0) RET(run_device(c));
    if (c.copied_out) {
        CK(cudaEventRecord(C->fields_in, C->copy)); // the last slab is on its way back
        CK(cudaStreamWaitEvent(st, C->fields_in, 0));
    } else {
        CK(cudaStreamWaitEvent(st, C->fields_in, 0));
        for (int f = 0; f < 6; ++f) {
            if (!grid->fields[f]) continue;
            const size_t b = (size_t)nvox * comps[f] * sizeof(double);
            CK(cudaMemcpyAsync(grid->fields[f], c.F[f], b, cudaMemcpyDeviceToHost, st));
        }
    }
    CK(cudaEventRecord(C->ev[7], st));
    CK(cudaEventSynchronize(C->ev[7]));
    if (o.stats) CK(cudaEventElapsedTime(&o.stats->ms_total, C->ev[0], C->ev[7]));
    return PSIB_OK;
}

int psib_voxels_batch(const psib_grid* grids, const psib_mesh* meshes, int nbatch, int mode, double refine_tolerance,
                      int refine_max_lvl, const psib_options* opt)
{
    g_err.clear();
    psib_options o = {};
    o.precision = PSIB_FP64;
    o.memory = PSIB_DEVICE;
    o.device = -1;
    if (opt) o = *opt;
    if (!grids || !meshes || nbatch <= 0) return fail(PSIB_ERR_ARG, "grids, meshes and nbatch > 0 are required");
    if (nbatch > 65535) return fail(PSIB_ERR_ARG, "at most 65535 cutouts per batch");
    if (o.memory != PSIB_DEVICE) return fail(PSIB_ERR_UNSUPPORTED, "a batch takes device memory (PSIB_DEVICE)");
    if (mode == PSIB_MODE_ANNIHILATION) return fail(PSIB_ERR_UNSUPPORTED, "a batch deposits density only");
    unsigned long long nvox = 0;
    long long nelem = 0;
    for (int b = 0; b < nbatch; ++b) {
        if (int r = validate(&grids[b], &meshes[b], mode, &o)) {
            g_err = "cutout " + std::to_string(b) + ": " + g_err;
            return r;
        }
        for (int f = 0; f < 6; ++f)
            if ((grids[b].fields[f] == nullptr) != (grids[0].fields[f] == nullptr))
                return fail(PSIB_ERR_ARG, "cutout %d: every grid of a batch must have the same fields", b);
        nvox += (unsigned long long)grids[b].n[0] * grids[b].n[1] * grids[b].n[2];
        nelem += meshes[b].nelem;
    }
    if (nvox >= (1ull << 32)) return fail(PSIB_ERR_ARG, "a batch of 2^32 voxels or more is not supported");
    if (nelem >= (1ll << 31)) return fail(PSIB_ERR_ARG, "a batch of 2^31 elements or more is not supported");
    if (o.refine_mode == PSIB_REFINE_STRETCH && !(refine_tolerance > 0.0))
        return fail(PSIB_ERR_ARG, "the stretch threshold must be positive");
    if (psib_device_count() <= 0) return fail(PSIB_ERR_NODEVICE, "no CUDA device is visible");
    int dev = 0;
    CK(cudaGetDevice(&dev));
    Ctx* C = nullptr;
    RET(get_ctx(dev, &C));
    Call c = {};
    c.grid = &grids[0];
    c.mesh = &meshes[0];
    c.nbatch = nbatch;
    c.grids = grids;
    c.meshes = meshes;
    c.refine_cell_given = o.refine_cell;
    c.reftol = refine_tolerance;
    c.maxlvl = refine_max_lvl > 6 ? 6 : (refine_max_lvl < 0 ? 0 : refine_max_lvl);
    c.precision = o.precision;
    c.deterministic = o.deterministic;
    c.refine_mode = o.refine_mode;
    c.queue_voxels = o.queue_voxels;
    c.capture = o.capture;
    c.order_cell_bits = o.order_cell_bits;
    c.C = C;
    c.stats = o.capture == 2 ? nullptr : o.stats;
    if (o.stats) *o.stats = psib_stats{};
    for (int f = 0; f < 6; ++f) c.F[f] = grids[0].fields[f];
    c.pos = meshes[0].pos;
    c.vel = meshes[0].vel;
    c.mass = meshes[0].mass;
    c.conn = meshes[0].connectivity;
    if (nelem == 0) return PSIB_OK;
    RET(enter_own_stream(*C, (cudaStream_t)o.stream));
    c.st = C->own;
    if (o.capture == 2) {
        const int r = run_capture(c);
        RET(leave_own_stream(*C, (cudaStream_t)o.stream));
        return r;
    }
    CK(cudaEventRecord(C->ev[0], c.st));
    const int r = run_device(c);
    RET(leave_own_stream(*C, (cudaStream_t)o.stream));
    RET(r);
    if (o.stats) {
        CK(cudaEventRecord(C->ev[7], c.st));
        CK(cudaEventSynchronize(C->ev[7]));
        CK(cudaEventElapsedTime(&o.stats->ms_total, C->ev[0], C->ev[7]));
    }
    return PSIB_OK;
}

int psib_capture_status(void)
{
    g_err.clear();
    if (psib_device_count() <= 0) return fail(PSIB_ERR_NODEVICE, "no CUDA device is visible");
    int dev = 0;
    CK(cudaGetDevice(&dev));
    Ctx* C = nullptr;
    RET(get_ctx(dev, &C));
    if (!C->small.p) return PSIB_OK;
    CK(cudaDeviceSynchronize());
    unsigned long long h[S_WORDS];
    CK(cudaMemcpy(h, C->small.p, sizeof(h), cudaMemcpyDeviceToHost));
    const unsigned zero = 0;
    CK(cudaMemcpy(C->small.p, &zero, sizeof(zero), cudaMemcpyHostToDevice));
    Call c = {};
    return check_status(c, h);
}

int psib_voxels_adjoint(const psib_grid* grad, const psib_mesh* mesh, double refine_tolerance, int refine_max_lvl,
                        double* grad_pos, double* grad_vel, double* grad_mass, const psib_options* opt)
{
    g_err.clear();
    psib_options o = {};
    o.precision = PSIB_FP64;
    o.memory = PSIB_HOST;
    o.device = -1;
    if (opt) o = *opt;
    RET(validate(grad, mesh, PSIB_MODE_DENSITY, &o));
    for (int f = 1; f < 6; ++f)
        if (grad->fields[f])
            return fail(PSIB_ERR_UNSUPPORTED, "the adjoint takes the gradient of field m only");
    if (!grad_pos && mesh->nelem > 0) return fail(PSIB_ERR_ARG, "grad_pos is required");
    (void)grad_vel; // the density does not depend on the velocities
    if (psib_device_count() <= 0) return fail(PSIB_ERR_NODEVICE, "no CUDA device is visible");
    int dev = o.device;
    if (o.memory == PSIB_DEVICE || dev < 0) CK(cudaGetDevice(&dev));
    CK(cudaSetDevice(dev));
    Ctx* C = nullptr;
    RET(get_ctx(dev, &C));

    Call c = {};
    c.grid = grad;
    c.mesh = mesh;
    c.reftol = refine_tolerance;
    c.maxlvl = refine_max_lvl > 6 ? 6 : (refine_max_lvl < 0 ? 0 : refine_max_lvl);
    c.precision = PSIB_FP64;
    c.C = C;
    c.stats = o.stats;
    c.adjoint = true;
    if (o.stats) *o.stats = psib_stats{};
    if (mesh->nelem == 0) return PSIB_OK;

    const long long nvox = (long long)grad->n[0] * grad->n[1] * grad->n[2];
    if (o.memory == PSIB_DEVICE) {
        c.st = (cudaStream_t)o.stream;
        c.F[0] = grad->fields[0];
        c.pos = mesh->pos;
        c.vel = mesh->vel;
        c.mass = mesh->mass;
        c.conn = mesh->connectivity;
        c.gpos = grad_pos;
        c.gmass = grad_mass;
        CK(cudaEventRecord(C->ev[0], c.st));
        RET(run_device(c));
        if (o.stats) {
            CK(cudaEventRecord(C->ev[7], c.st));
            CK(cudaEventSynchronize(C->ev[7]));
            CK(cudaEventElapsedTime(&o.stats->ms_total, C->ev[0], C->ev[7]));
        }
        return PSIB_OK;
    }
    cudaStream_t st = C->own;
    c.st = st;
    CK(cudaEventRecord(C->ev[0], st));
    RET(copy_mesh_in(c, *C, *mesh, st));
    RET(ensure(C->hfield[0], (size_t)nvox * sizeof(double)));
    CK(cudaMemcpyAsync(C->hfield[0].p, grad->fields[0], (size_t)nvox * sizeof(double), cudaMemcpyHostToDevice, st));
    c.F[0] = C->hfield[0].as<double>();
    const size_t gpb = (size_t)mesh->npart * 3 * sizeof(double);
    RET(ensure(C->hgpos, gpb));
    CK(cudaMemcpyAsync(C->hgpos.p, grad_pos, gpb, cudaMemcpyHostToDevice, st));
    c.gpos = C->hgpos.as<double>();
    if (grad_mass) {
        RET(ensure(C->hgmass, (size_t)mesh->nelem * sizeof(double)));
        CK(cudaMemcpyAsync(C->hgmass.p, grad_mass, (size_t)mesh->nelem * sizeof(double), cudaMemcpyHostToDevice, st));
        c.gmass = C->hgmass.as<double>();
    }
    RET(run_device(c));
    CK(cudaMemcpyAsync(grad_pos, c.gpos, gpb, cudaMemcpyDeviceToHost, st));
    if (grad_mass)
        CK(cudaMemcpyAsync(grad_mass, c.gmass, (size_t)mesh->nelem * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaEventRecord(C->ev[7], st));
    CK(cudaEventSynchronize(C->ev[7]));
    if (o.stats) CK(cudaEventElapsedTime(&o.stats->ms_total, C->ev[0], C->ev[7]));
    return PSIB_OK;
}

int psib_voxels_adjoint_fields(const psib_grid* grad, const psib_grid* fwd, const psib_mesh* mesh,
                               double refine_tolerance, int refine_max_lvl, double* grad_pos, double* grad_vel,
                               double* grad_mass, const psib_options* opt)
{
    g_err.clear();
    psib_options o = {};
    o.precision = PSIB_FP64;
    o.memory = PSIB_DEVICE;
    o.device = -1;
    if (opt) o = *opt;
    if (!grad || !fwd) return fail(PSIB_ERR_ARG, "grad and fwd are required");
    RET(validate(fwd, mesh, PSIB_MODE_DENSITY, &o));
    for (int i = 0; i < 3; ++i)
        if (grad->n[i] != fwd->n[i] || grad->window[0][i] != fwd->window[0][i] ||
            grad->window[1][i] != fwd->window[1][i])
            return fail(PSIB_ERR_ARG, "grad and fwd must describe the same grid");
    static const char* names[6] = {"m", "x", "v", "xx", "xv", "vv"};
    for (int f = 0; f < 6; ++f)
        if (grad->fields[f] && !fwd->fields[f])
            return fail(PSIB_ERR_ARG, "the gradient of field %s needs the forward field %s", names[f], names[f]);
    if ((fwd->fields[PSIB_XX] && !fwd->fields[PSIB_X]) || (fwd->fields[PSIB_VV] && !fwd->fields[PSIB_V]) ||
        (fwd->fields[PSIB_XV] && !(fwd->fields[PSIB_X] && fwd->fields[PSIB_V])))
        return fail(PSIB_ERR_ARG, "the forward second moments need their first moments (xx: x, vv: v, xv: x and v)");
    if (o.memory != PSIB_DEVICE) return fail(PSIB_ERR_UNSUPPORTED, "psib_voxels_adjoint_fields takes device memory");
    if (!grad_pos && mesh->nelem > 0) return fail(PSIB_ERR_ARG, "grad_pos is required");
    if (psib_device_count() <= 0) return fail(PSIB_ERR_NODEVICE, "no CUDA device is visible");
    int dev = 0;
    CK(cudaGetDevice(&dev));
    Ctx* C = nullptr;
    RET(get_ctx(dev, &C));
    if (o.stats) *o.stats = psib_stats{};
    if (mesh->nelem == 0) return PSIB_OK;
    const long long nvox = (long long)fwd->n[0] * fwd->n[1] * fwd->n[2];
    cudaStream_t st = (cudaStream_t)o.stream;
    RET(ensure(C->adjcoef, (size_t)nvox * ADJ_NCOEF * sizeof(double)));
    AdjCoefArgs ac = {};
    for (int f = 0; f < 6; ++f) {
        ac.F[f] = fwd->fields[f];
        ac.G[f] = grad->fields[f];
    }
    ac.coef = C->adjcoef.as<double>();
    ac.nvox = nvox;
    CK(launch_adj_coeffs(ac, st));

    Call c = {};
    c.grid = fwd;
    c.mesh = mesh;
    c.reftol = refine_tolerance;
    c.maxlvl = refine_max_lvl > 6 ? 6 : (refine_max_lvl < 0 ? 0 : refine_max_lvl);
    c.precision = PSIB_FP64;
    c.C = C;
    c.stats = o.stats;
    c.adjoint = true;
    c.adj_coef = C->adjcoef.as<double>();
    c.st = st;
    c.pos = mesh->pos;
    c.vel = mesh->vel;
    c.mass = mesh->mass;
    c.conn = mesh->connectivity;
    c.gpos = grad_pos;
    c.gvel = grad_vel;
    c.gmass = grad_mass;
    CK(cudaEventRecord(C->ev[0], st));
    RET(run_device(c));
    if (o.stats) {
        CK(cudaEventRecord(C->ev[7], st));
        CK(cudaEventSynchronize(C->ev[7]));
        CK(cudaEventElapsedTime(&o.stats->ms_total, C->ev[0], C->ev[7]));
    }
    return PSIB_OK;
}

} // extern "C"
