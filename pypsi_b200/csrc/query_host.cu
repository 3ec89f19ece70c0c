// query_host.cu -- the host side of element queries and phase-space samples
// (psib_query_elements, psib_sample_vdf) and of the persistent element index
// (psib_index_*), over the cell index of annihilation_host.cu.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "pipeline_host.h"

using namespace psib;
using namespace psib::host;

namespace {

// ---- element queries and phase-space samples ----

// A query call: device, context, stream and the mesh in device memory (copied
// in for host-memory calls; device-memory calls run on the library's stream
// fenced to the caller's).
struct QueryCall {
    Call c;
    Ctx* C = nullptr;
    bool host = true;
    cudaStream_t user = nullptr;
};

int query_begin(QueryCall& q, const psib_mesh* mesh, const psib_options* opt)
{
    g_err.clear();
    RET(validate_mesh(mesh));
    psib_options o = {};
    o.memory = PSIB_HOST;
    o.device = -1;
    if (opt) o = *opt;
    if (o.memory != PSIB_HOST && o.memory != PSIB_DEVICE) return fail(PSIB_ERR_ARG, "invalid memory kind %d", o.memory);
    if (psib_device_count() <= 0) return fail(PSIB_ERR_NODEVICE, "no CUDA device is visible");
    int dev = o.device;
    if (o.memory == PSIB_DEVICE || dev < 0) CK(cudaGetDevice(&dev));
    CK(cudaSetDevice(dev));
    RET(get_ctx(dev, &q.C));
    q.host = o.memory == PSIB_HOST;
    q.c = Call{};
    q.c.mesh = mesh;
    q.c.C = q.C;
    q.c.st = q.C->own;
    if (q.host) {
        if (mesh->nelem > 0) RET(copy_mesh_in(q.c, *q.C, *mesh, q.c.st));
    } else {
        q.user = (cudaStream_t)o.stream;
        RET(enter_own_stream(*q.C, q.user));
        q.c.pos = mesh->pos;
        q.c.vel = mesh->vel;
        q.c.mass = mesh->mass;
        q.c.conn = mesh->connectivity;
    }
    return PSIB_OK;
}

int query_end(QueryCall& q, int rc)
{
    if (!q.host && q.C) {
        const int r = leave_own_stream(*q.C, q.user);
        if (rc == PSIB_OK) rc = r;
    }
    if (rc == PSIB_OK) CK(cudaStreamSynchronize(q.c.st));
    return rc;
}

// The kept elements (cull against `window`) and their unwrapped boxes.
int query_elements_stage(QueryCall& q, const double (*window)[3], double reftol, AnnArgs& aa, unsigned long long* sm)
{
    Ctx& C = *q.C;
    const psib_mesh& m = *q.c.mesh;
    const long long ne = m.nelem;
    cudaStream_t st = q.c.st;
    psib_grid gw = {};
    for (int i = 0; i < 3; ++i) {
        gw.n[i] = 1;
        gw.window[0][i] = window[0][i];
        gw.window[1][i] = window[1][i];
        gw.d[i] = 1.0;
    }
    MeshDev md = mesh_dev(m, gw, q.c.pos, q.c.vel, q.c.mass, q.c.conn, 1.0, nullptr);
    md.ptol2 = reftol * reftol; // psi_tet_buffer_init(&tetbuf, reftol, ...): the tolerance itself (src/cpsi.c:198)
    RET(ensure(C.a_cnt, (size_t)2 * (ne + 1) * sizeof(int)));
    RET(ensure(C.a_ebox, (size_t)(ne > 0 ? ne : 1) * 6 * sizeof(double)));
    AnnTessArgs ta = {};
    ta.m = md;
    ta.g = grid_dev(gw);
    ta.cnt_a = C.a_cnt.as<int>();
    ta.cnt_b = ta.cnt_a + (ne + 1);
    ta.ebox = C.a_ebox.as<double>();
    ta.status = (unsigned*)&sm[S_STATUS];
    if (ne > 0) CK(launch_elem_boxes(ta, st));
    aa = AnnArgs{};
    aa.nelem = ne;
    aa.ebox = ta.ebox;
    aa.cnt_a = ta.cnt_a;
    aa.cnt_b = ta.cnt_b;
    aa.status = ta.status;
    q.c.reftol = reftol;
    return PSIB_OK;
}

// A device buffer of `bytes` holding the caller's array (copied in for host-memory calls).
int query_input(QueryCall& q, DevBuf& b, const void* src, size_t bytes, const void** dst)
{
    if (!q.host) {
        *dst = src;
        return PSIB_OK;
    }
    RET(ensure(b, bytes > 0 ? bytes : 16));
    if (bytes) CK(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, q.c.st));
    *dst = b.p;
    return PSIB_OK;
}

int query_output(QueryCall& q, void* dst, const void* src, size_t bytes)
{
    if (!bytes) return PSIB_OK;
    CK(cudaMemcpyAsync(dst, src, bytes, q.host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, q.c.st));
    return PSIB_OK;
}

int sort_keys(Ctx& C, unsigned long long* in, unsigned long long* out, long long n, int bits, cudaStream_t st)
{
    if (n >= (1ll << 31)) return fail(PSIB_ERR_OVERFLOW, "too many query results (%lld)", n);
    size_t tb = 0;
    CK(cub::DeviceRadixSort::SortKeys(nullptr, tb, in, out, (int)n, 0, bits, st));
    RET(ensure(C.cub_tmp, tb));
    CK(cub::DeviceRadixSort::SortKeys(C.cub_tmp.p, tb, in, out, (int)n, 0, bits, st));
    return PSIB_OK;
}

int query_status(QueryCall& q, unsigned long long* sm)
{
    unsigned long long h[S_WORDS];
    CK(cudaMemcpyAsync(h, sm, sizeof(h), cudaMemcpyDeviceToHost, q.c.st));
    CK(cudaStreamSynchronize(q.c.st));
    return check_status(q.c, h);
}

int query_from_boxes(QueryCall& q, AnnArgs& aa, unsigned long long* sm, const double* boxes, long long nboxes,
                     long long* offsets, int* elements, long long capacity);
int vdf_from_index(QueryCall& q, AnnArgs& aa, long long kept, unsigned long long* sm, const double* points,
                   long long npoints, double reftol, int maxlvl, long long* offsets, double* rho, double* vel,
                   long long capacity);
int vdf_one_point(QueryCall& q, AnnArgs& aa, long long kept, unsigned long long* sm, double reftol, int maxlvl,
                  long long* offsets, double* rho, double* vel, long long capacity);

int query_elements_impl(QueryCall& q, const double (*window)[3], const double* boxes, long long nboxes,
                        long long* offsets, int* elements, long long capacity)
{
    Ctx& C = *q.C;
    cudaStream_t st = q.c.st;
    RET(ensure(C.small, S_WORDS * 8));
    unsigned long long* sm = C.small.as<unsigned long long>();
    CK(cudaMemsetAsync(sm, 0, S_WORDS * 8, st));
    AnnArgs aa;
    RET(query_elements_stage(q, window, 1.0, aa, sm));
    return query_from_boxes(q, aa, sm, boxes, nboxes, offsets, elements, capacity);
}

// Box queries over the kept element boxes of aa (cnt_a flags, ebox).
int query_from_boxes(QueryCall& q, AnnArgs& aa, unsigned long long* sm, const double* boxes, long long nboxes,
                     long long* offsets, int* elements, long long capacity)
{
    Ctx& C = *q.C;
    cudaStream_t st = q.c.st;
    const void* qin = nullptr;
    RET(query_input(q, C.q_in, boxes, (size_t)nboxes * 6 * sizeof(double), &qin));
    aa.qry = (const double*)qin;
    aa.nq = nboxes;
    RET(ensure(C.q_cnt, (size_t)(nboxes + 1) * sizeof(long long)));
    RET(ensure(C.q_off, (size_t)(nboxes + 1) * sizeof(long long)));
    RET(ensure(C.small, S_WORDS * 8));
    aa.q_cnt = C.q_cnt.as<long long>();
    CK(cudaMemsetAsync(aa.q_cnt, 0, (size_t)(nboxes + 1) * sizeof(long long), st));
    if (nboxes > 0 && aa.nelem > 0) CK(launch_query_boxes(aa, false, st));
    RET(excl_scan(C, aa.q_cnt, C.q_off.as<long long>(), nboxes + 1, st));
    long long total = 0;
    RET(read_dev(C.q_off.as<long long>() + nboxes, total, st));
    RET(query_status(q, sm));
    RET(query_output(q, offsets, C.q_off.p, (size_t)(nboxes + 1) * sizeof(long long)));
    if (!elements) return PSIB_OK;
    if (capacity < total)
        return fail(PSIB_ERR_OVERFLOW, "the output holds %lld elements, the queries found %lld", capacity, total);
    if (total == 0) return PSIB_OK;
    RET(ensure(C.q_key, (size_t)total * 8));
    RET(ensure(C.q_key_s, (size_t)total * 8));
    aa.q_key = C.q_key.as<unsigned long long>();
    aa.q_n = &sm[S_RECN];
    CK(cudaMemsetAsync(aa.q_n, 0, 8, st));
    CK(launch_query_boxes(aa, true, st));
    RET(sort_keys(C, aa.q_key, C.q_key_s.as<unsigned long long>(), total, 32 + bits_for((unsigned long long)nboxes + 1),
                  st));
    int* out = elements;
    if (q.host) {
        RET(ensure(C.q_out, (size_t)total * sizeof(int)));
        out = C.q_out.as<int>();
    }
    CK(launch_keys_elem(C.q_key_s.as<unsigned long long>(), total, out, st));
    if (q.host) RET(query_output(q, elements, out, (size_t)total * sizeof(int)));
    return query_status(q, sm);
}

int sample_vdf_impl(QueryCall& q, const double (*window)[3], const double* points, long long npoints, double reftol,
                    int maxlvl, long long* offsets, double* rho, double* vel, long long capacity)
{
    Ctx& C = *q.C;
    cudaStream_t st = q.c.st;
    RET(ensure(C.small, S_WORDS * 8));
    unsigned long long* sm = C.small.as<unsigned long long>();
    CK(cudaMemsetAsync(sm, 0, S_WORDS * 8, st));
    AnnArgs aa;
    RET(query_elements_stage(q, window, reftol, aa, sm));
    long long klaunch = 0, kept = 0;
    if (aa.nelem > 0) RET(build_cells(C, aa, st, klaunch, kept));
    return vdf_from_index(q, aa, kept, sm, points, npoints, reftol, maxlvl, offsets, rho, vel, capacity);
}

// One point in host memory (the drop-in PSI.VDF call): one thread walks the
// point's cell and writes the samples that fit `capacity`; one copy brings
// back their number and the samples.
int vdf_one_point(QueryCall& q, AnnArgs& aa, long long kept, unsigned long long* sm, double reftol, int maxlvl,
                  long long* offsets, double* rho, double* vel, long long capacity)
{
    Ctx& C = *q.C;
    cudaStream_t st = q.c.st;
    const psib_mesh& m = *q.c.mesh;
    VdfArgs va = {};
    va.m = mesh_dev(m, psib_grid{}, q.c.pos, q.c.vel, q.c.mass, q.c.conn, 1.0, nullptr);
    va.m.ptol2 = reftol * reftol;
    va.max_lvl = maxlvl > 6 ? 6 : (maxlvl < 0 ? 0 : maxlvl);
    va.quad = m.elemtype == 27;
    va.points = aa.qry;
    va.status = aa.status;
    const long long cap = (rho && vel) ? (capacity > 0 ? capacity : 0) : 0;
    RET(ensure(C.s_rho, (size_t)(cap > 0 ? cap : 1) * sizeof(double)));
    RET(ensure(C.s_vel, (size_t)(cap > 0 ? cap : 1) * 3 * sizeof(double)));
    va.rho = C.s_rho.as<double>();
    va.vel = C.s_vel.as<double>();
    CK(cudaMemsetAsync(&sm[S_RECN], 0, 8, st));
    if (kept > 0) CK(launch_vdf_point(va, aa, &sm[S_RECN], cap, st));
    unsigned long long h[S_WORDS];
    CK(cudaMemcpyAsync(h, sm, sizeof(h), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    RET(check_status(q.c, h));
    const long long total = (long long)h[S_RECN];
    offsets[0] = 0;
    offsets[1] = total;
    if (!rho || !vel) return PSIB_OK;
    if (capacity < total)
        return fail(PSIB_ERR_OVERFLOW, "the output holds %lld samples, the points have %lld", capacity, total);
    if (total > 0) {
        CK(cudaMemcpyAsync(rho, va.rho, (size_t)total * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(vel, va.vel, (size_t)total * 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    return PSIB_OK;
}

// Samples at the points through the cell index of aa (kept elements, their
// boxes, cells and runs), the mesh of q.
int vdf_from_index(QueryCall& q, AnnArgs& aa, long long kept, unsigned long long* sm, const double* points,
                   long long npoints, double reftol, int maxlvl, long long* offsets, double* rho, double* vel,
                   long long capacity)
{
    Ctx& C = *q.C;
    cudaStream_t st = q.c.st;
    const psib_mesh& m = *q.c.mesh;
    const void* qin = nullptr;
    RET(query_input(q, C.q_in, points, (size_t)npoints * 3 * sizeof(double), &qin));
    aa.qry = (const double*)qin;
    aa.nq = npoints;
    if (npoints == 1 && q.host)
        return vdf_one_point(q, aa, kept, sm, reftol, maxlvl, offsets, rho, vel, capacity);
    // (point, element) pairs: every kept element whose box contains the point
    RET(ensure(C.q_cnt, (size_t)(npoints + 1) * sizeof(long long)));
    RET(ensure(C.q_off, (size_t)(npoints + 1) * sizeof(long long)));
    aa.q_cnt = C.q_cnt.as<long long>();
    CK(cudaMemsetAsync(aa.q_cnt, 0, (size_t)(npoints + 1) * sizeof(long long), st));
    if (kept > 0 && npoints > 0) CK(launch_query_points(aa, false, st));
    RET(excl_scan(C, aa.q_cnt, C.q_off.as<long long>(), npoints + 1, st));
    aa.q_off = C.q_off.as<long long>();
    long long npair = 0;
    RET(read_dev(aa.q_off + npoints, npair, st));
    RET(ensure(C.q_key, (size_t)(npair > 0 ? npair : 1) * 8));
    aa.q_key = C.q_key.as<unsigned long long>();
    if (npair > 0) CK(launch_query_points(aa, true, st)); // keys come out sorted: point, element descending
    // samples per pair, in pair order (point, element descending, tet)
    VdfArgs va = {};
    va.m = mesh_dev(m, psib_grid{}, q.c.pos, q.c.vel, q.c.mass, q.c.conn, 1.0, nullptr);
    va.m.ptol2 = reftol * reftol;
    va.max_lvl = maxlvl > 6 ? 6 : (maxlvl < 0 ? 0 : maxlvl);
    va.quad = m.elemtype == 27;
    va.points = aa.qry;
    va.pairs = aa.q_key;
    va.npair = npair;
    va.status = (unsigned*)&sm[S_STATUS];
    RET(ensure(C.s_cnt, (size_t)(npair + 1) * sizeof(long long)));
    RET(ensure(C.s_off, (size_t)(npair + 1) * sizeof(long long)));
    va.cnt = C.s_cnt.as<long long>();
    CK(cudaMemsetAsync(va.cnt, 0, (size_t)(npair + 1) * sizeof(long long), st));
    if (npair > 0) CK(launch_vdf_samples(va, false, st));
    RET(excl_scan(C, va.cnt, C.s_off.as<long long>(), npair + 1, st));
    va.off = C.s_off.as<long long>();
    long long total = 0;
    RET(read_dev(va.off + npair, total, st));
    // each point's first sample: the sample offset of its first pair
    RET(ensure(C.s_offs, (size_t)(npoints + 1) * sizeof(long long)));
    CK(launch_gather_ll(va.off, aa.q_off, npoints + 1, C.s_offs.as<long long>(), st));
    RET(query_status(q, sm));
    RET(query_output(q, offsets, C.s_offs.p, (size_t)(npoints + 1) * sizeof(long long)));
    if (!rho || !vel) return PSIB_OK;
    if (capacity < total)
        return fail(PSIB_ERR_OVERFLOW, "the output holds %lld samples, the points have %lld", capacity, total);
    if (total == 0) return PSIB_OK;
    if (q.host) {
        RET(ensure(C.s_rho, (size_t)total * sizeof(double)));
        RET(ensure(C.s_vel, (size_t)total * 3 * sizeof(double)));
        va.rho = C.s_rho.as<double>();
        va.vel = C.s_vel.as<double>();
    } else {
        va.rho = rho;
        va.vel = vel;
    }
    CK(launch_vdf_samples(va, true, st));
    if (q.host) {
        RET(query_output(q, rho, va.rho, (size_t)total * sizeof(double)));
        RET(query_output(q, vel, va.vel, (size_t)total * 3 * sizeof(double)));
    }
    return query_status(q, sm);
}

} // namespace

// ---- a persistent element index (PSI.RStarTree) ----

// The mesh (device copies), its kept elements' boxes and the cell index over
// them, built once; later queries and samples reuse them.
struct psib_index {
    int device = 0;
    psib_mesh mesh = {}; // device pointers into the buffers below
    psib::AnnArgs aa = {}; // kept flags, boxes, cells and runs, pointing into the buffers below
    long long kept = 0;
    DevBuf pos, vel, mass, conn, ebox, cnt, reg_elem, run_key, run_off, run_cnt;
};

namespace {

int copy_dev(DevBuf& dst, const void* src, size_t bytes, cudaStream_t st)
{
    RET(ensure(dst, bytes));
    if (bytes && src) CK(cudaMemcpyAsync(dst.p, src, bytes, cudaMemcpyDeviceToDevice, st));
    return PSIB_OK;
}

void free_index(psib_index* ix)
{
    if (!ix) return;
    for (DevBuf* b : {&ix->pos, &ix->vel, &ix->mass, &ix->conn, &ix->ebox, &ix->cnt, &ix->reg_elem, &ix->run_key,
                      &ix->run_off, &ix->run_cnt})
        if (b->p) cudaFree(b->p);
    delete ix;
}

int index_fill(QueryCall& q, const double (*window)[3], psib_index* ix)
{
    Ctx& C = *q.C;
    cudaStream_t st = q.c.st;
    const psib_mesh& m = *q.c.mesh;
    RET(ensure(C.small, S_WORDS * 8));
    unsigned long long* sm = C.small.as<unsigned long long>();
    CK(cudaMemsetAsync(sm, 0, S_WORDS * 8, st));
    psib::AnnArgs aa;
    RET(query_elements_stage(q, window, 1.0, aa, sm));
    long long klaunch = 0, kept = 0;
    if (aa.nelem > 0) RET(build_cells(C, aa, st, klaunch, kept));
    RET(query_status(q, sm));
    const size_t np = (size_t)m.npart, ne = (size_t)m.nelem;
    RET(copy_dev(ix->pos, q.c.pos, np * 24, st));
    if (q.c.vel) RET(copy_dev(ix->vel, q.c.vel, np * 24, st));
    if (q.c.mass) RET(copy_dev(ix->mass, q.c.mass, ne * 8, st));
    if (q.c.conn) RET(copy_dev(ix->conn, q.c.conn, ne * (size_t)m.elemtype * 4, st));
    RET(copy_dev(ix->ebox, aa.ebox, ne * 48, st));
    RET(copy_dev(ix->cnt, aa.cnt_a, 2 * (ne + 1) * sizeof(int), st));
    if (kept > 0) {
        RET(copy_dev(ix->reg_elem, aa.reg_elem, (size_t)aa.nreg * sizeof(int), st));
        RET(copy_dev(ix->run_key, aa.run_key, (size_t)aa.nruns * 8, st));
        RET(copy_dev(ix->run_off, aa.run_off, (size_t)aa.nruns * 8, st));
        RET(copy_dev(ix->run_cnt, aa.run_cnt, (size_t)aa.nruns * sizeof(int), st));
    }
    CK(cudaStreamSynchronize(st));
    ix->device = C.device;
    ix->kept = kept;
    ix->mesh = m;
    ix->mesh.pos = ix->pos.as<double>();
    ix->mesh.vel = q.c.vel ? ix->vel.as<double>() : nullptr;
    ix->mesh.mass = q.c.mass ? ix->mass.as<double>() : nullptr;
    ix->mesh.connectivity = q.c.conn ? ix->conn.as<int>() : nullptr;
    psib::AnnArgs& a = ix->aa;
    a = psib::AnnArgs{};
    a.nelem = aa.nelem;
    a.cg = aa.cg;
    a.nreg = aa.nreg;
    a.nruns = aa.nruns;
    a.ebox = ix->ebox.as<double>();
    a.cnt_a = ix->cnt.as<int>();
    a.cnt_b = ix->cnt.as<int>() + (ne + 1);
    a.reg_elem = ix->reg_elem.as<int>();
    a.run_key = ix->run_key.as<unsigned long long>();
    a.run_off = ix->run_off.as<long long>();
    a.run_cnt = ix->run_cnt.as<int>();
    return PSIB_OK;
}

// A call on an index: its device and mesh, points and outputs in the memory options->memory names.
int index_begin(QueryCall& q, psib_index* ix, const psib_options* opt)
{
    g_err.clear();
    if (!ix) return fail(PSIB_ERR_ARG, "index is required");
    psib_options o = {};
    o.memory = PSIB_HOST;
    if (opt) o = *opt;
    if (o.memory != PSIB_HOST && o.memory != PSIB_DEVICE) return fail(PSIB_ERR_ARG, "invalid memory kind %d", o.memory);
    if (psib_device_count() <= 0) return fail(PSIB_ERR_NODEVICE, "no CUDA device is visible");
    CK(cudaSetDevice(ix->device));
    RET(get_ctx(ix->device, &q.C));
    q.host = o.memory == PSIB_HOST;
    q.c = Call{};
    q.c.mesh = &ix->mesh;
    q.c.C = q.C;
    q.c.st = q.C->own;
    q.c.pos = ix->mesh.pos;
    q.c.vel = ix->mesh.vel;
    q.c.mass = ix->mesh.mass;
    q.c.conn = ix->mesh.connectivity;
    if (!q.host) {
        q.user = (cudaStream_t)o.stream;
        RET(enter_own_stream(*q.C, q.user));
    }
    return PSIB_OK;
}

unsigned long long* index_status(QueryCall& q, psib::AnnArgs& aa, int& rc)
{
    rc = ensure(q.C->small, S_WORDS * 8);
    if (rc) return nullptr;
    unsigned long long* sm = q.C->small.as<unsigned long long>();
    if (cudaMemsetAsync(sm, 0, S_WORDS * 8, q.c.st) != cudaSuccess) {
        rc = fail(PSIB_ERR_CUDA, "cudaMemsetAsync failed");
        return nullptr;
    }
    aa.status = (unsigned*)&sm[S_STATUS];
    return sm;
}

} // namespace

extern "C" {

int psib_query_elements(const psib_mesh* mesh, const double window[2][3], const double* boxes, long long nboxes,
                        long long* offsets, int* elements, long long capacity, const psib_options* opt)
{
    if (!window || !offsets || nboxes < 0 || (nboxes > 0 && !boxes))
        return fail(PSIB_ERR_ARG, "window, offsets and nboxes >= 0 boxes are required");
    if (nboxes >= (1ll << 31)) return fail(PSIB_ERR_ARG, "at most 2^31 - 1 query boxes");
    QueryCall q;
    RET(query_begin(q, mesh, opt));
    return query_end(q, query_elements_impl(q, window, boxes, nboxes, offsets, elements, capacity));
}

int psib_sample_vdf(const psib_mesh* mesh, const double window[2][3], const double* points, long long npoints,
                    double refine_tolerance, int refine_max_lvl, long long* offsets, double* rho, double* vel,
                    long long capacity, const psib_options* opt)
{
    if (!window || !offsets || npoints < 0 || (npoints > 0 && !points))
        return fail(PSIB_ERR_ARG, "window, offsets and npoints >= 0 points are required");
    if (npoints >= (1ll << 31)) return fail(PSIB_ERR_ARG, "at most 2^31 - 1 sample points");
    QueryCall q;
    RET(query_begin(q, mesh, opt));
    return query_end(q, sample_vdf_impl(q, window, points, npoints, refine_tolerance, refine_max_lvl, offsets, rho,
                                        vel, capacity));
}

int psib_index_create(const psib_mesh* mesh, const double window[2][3], psib_index** index, const psib_options* opt)
{
    if (!index || !window) return fail(PSIB_ERR_ARG, "index and window are required");
    *index = nullptr;
    QueryCall q;
    RET(query_begin(q, mesh, opt));
    psib_index* ix = new psib_index();
    const int rc = query_end(q, index_fill(q, window, ix));
    if (rc != PSIB_OK) {
        free_index(ix);
        return rc;
    }
    *index = ix;
    return PSIB_OK;
}

int psib_index_query(psib_index* index, const double* boxes, long long nboxes, long long* offsets, int* elements,
                     long long capacity, const psib_options* opt)
{
    if (!offsets || nboxes < 0 || (nboxes > 0 && !boxes))
        return fail(PSIB_ERR_ARG, "offsets and nboxes >= 0 boxes are required");
    if (nboxes >= (1ll << 31)) return fail(PSIB_ERR_ARG, "at most 2^31 - 1 query boxes");
    QueryCall q;
    RET(index_begin(q, index, opt));
    psib::AnnArgs aa = index->aa;
    int rc = PSIB_OK;
    unsigned long long* sm = index_status(q, aa, rc);
    if (rc == PSIB_OK) rc = query_from_boxes(q, aa, sm, boxes, nboxes, offsets, elements, capacity);
    return query_end(q, rc);
}

int psib_index_sample_vdf(psib_index* index, const double* points, long long npoints, double refine_tolerance,
                          int refine_max_lvl, long long* offsets, double* rho, double* vel, long long capacity,
                          const psib_options* opt)
{
    if (!offsets || npoints < 0 || (npoints > 0 && !points))
        return fail(PSIB_ERR_ARG, "offsets and npoints >= 0 points are required");
    if (npoints >= (1ll << 31)) return fail(PSIB_ERR_ARG, "at most 2^31 - 1 sample points");
    QueryCall q;
    RET(index_begin(q, index, opt));
    psib::AnnArgs aa = index->aa;
    int rc = PSIB_OK;
    unsigned long long* sm = index_status(q, aa, rc);
    if (rc == PSIB_OK)
        rc = vdf_from_index(q, aa, index->kept, sm, points, npoints, refine_tolerance, refine_max_lvl, offsets, rho,
                            vel, capacity);
    return query_end(q, rc);
}

void psib_index_destroy(psib_index* index)
{
    if (!index) return;
    int cur = 0;
    const bool have = cudaGetDevice(&cur) == cudaSuccess;
    if (cudaSetDevice(index->device) == cudaSuccess) cudaDeviceSynchronize();
    free_index(index);
    if (have) cudaSetDevice(cur);
    cudaGetLastError();
}

} // extern "C"
