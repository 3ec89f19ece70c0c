// annihilation_host.cu -- the host side of annihilation mode (psib_voxels with
// PSIB_MODE_ANNIHILATION): the cell index over the element boxes that the pair
// search and the element queries share, and the stages of one call
// (annihilation.cu holds the kernels).
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pipeline_host.h"
#include "psib_device.cuh"

namespace psib {
namespace host {

double from_ord(unsigned long long o)
{
    const unsigned long long b = (o >> 63) ? (o & 0x7FFFFFFFFFFFFFFFull) : ~o;
    double x;
    memcpy(&x, &b, 8);
    return x;
}

// The cell index over the kept element boxes (aa.nelem, aa.ebox and the kept
// flags aa.cnt_a / aa.cnt_b set): a uniform grid of cells about one mean
// element box wide (at most 1024 per axis); every kept element registered in
// the cells its box covers, sorted by cell; each registration's cell run
// (aa.run_lo / run_hi) and the runs themselves (aa.run_key / run_off /
// run_cnt, aa.nruns).  kept = the number of kept elements (0: no index).
int build_cells(Ctx& C, AnnArgs& aa, cudaStream_t st, long long& klaunch, long long& kept)
{
    const long long ne = aa.nelem;
    RET(ensure(C.a_stats, 16 * 8));
    CK(cudaMemsetAsync(C.a_stats.p, 0xFF, 3 * 8, st));
    CK(cudaMemsetAsync(C.a_stats.as<char>() + 24, 0, 13 * 8, st));
    unsigned long long* bs = C.a_stats.as<unsigned long long>();
    CK(launch_ann_box_stats(aa, bs, (double*)(bs + 8), st));
    klaunch++;
    unsigned long long hb[16];
    CK(cudaMemcpyAsync(hb, bs, sizeof(hb), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    kept = (long long)hb[6];
    if (kept == 0) return PSIB_OK;
    long long ncell = 1;
    for (int i = 0; i < 3; ++i) {
        const double lo = from_ord(hb[i]), hi = from_ord(hb[3 + i]);
        double ext;
        memcpy(&ext, &hb[8 + i], 8);
        const double range = hi - lo;
        // cells about one mean element box wide, at most 1024 per axis
        double h = ext / (double)kept;
        if (!(h >= range / 1024.0)) h = range / 1024.0;
        if (!(h > 0.0) || !std::isfinite(h)) h = range > 0.0 && std::isfinite(range) ? range : 1.0;
        aa.cg.o[i] = std::isfinite(lo) ? lo : 0.0;
        aa.cg.h[i] = h;
        long long n = std::isfinite(range) ? (long long)(range / h) + 1 : 1;
        aa.cg.n[i] = n < 1 ? 1 : (n > 1024 ? 1024 : n);
        ncell *= aa.cg.n[i];
    }

    // ---- cell registrations, sorted by cell ----
    RET(ensure(C.a_reg_cnt, (size_t)(ne + 1) * sizeof(long long)));
    RET(ensure(C.a_reg_off, (size_t)(ne + 1) * sizeof(long long)));
    aa.reg_cnt = C.a_reg_cnt.as<long long>();
    CK(launch_ann_cells(aa, false, st));
    CK(cudaMemsetAsync(aa.reg_cnt + ne, 0, sizeof(long long), st));
    RET(excl_scan(C, aa.reg_cnt, C.a_reg_off.as<long long>(), ne + 1, st));
    long long nreg = 0;
    RET(read_dev(C.a_reg_off.as<long long>() + ne, nreg, st));
    if (nreg >= (1ll << 31)) return fail(PSIB_ERR_OVERFLOW, "too many cell registrations (%lld)", nreg);
    RET(ensure(C.a_reg_key, (size_t)nreg * 8));
    RET(ensure(C.a_reg_elem, (size_t)nreg * 4));
    RET(ensure(C.a_reg_key_s, (size_t)nreg * 8));
    RET(ensure(C.a_reg_elem_s, (size_t)nreg * 4));
    aa.reg_off = C.a_reg_off.as<long long>();
    aa.reg_key = C.a_reg_key.as<unsigned long long>();
    aa.reg_elem = C.a_reg_elem.as<int>();
    CK(launch_ann_cells(aa, true, st));
    klaunch += 2;
    {
        size_t tb = 0;
        const int cb = bits_for((unsigned long long)ncell);
        CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, aa.reg_key, C.a_reg_key_s.as<unsigned long long>(), aa.reg_elem,
                                           C.a_reg_elem_s.as<int>(), (int)nreg, 0, cb, st));
        RET(ensure(C.cub_tmp, tb));
        CK(cub::DeviceRadixSort::SortPairs(C.cub_tmp.p, tb, aa.reg_key, C.a_reg_key_s.as<unsigned long long>(),
                                           aa.reg_elem, C.a_reg_elem_s.as<int>(), (int)nreg, 0, cb, st));
    }
    aa.reg_key = C.a_reg_key_s.as<unsigned long long>();
    aa.reg_elem = C.a_reg_elem_s.as<int>();
    aa.nreg = nreg;
    // each registration's cell run
    RET(ensure(C.a_run_key, (size_t)nreg * 8));
    RET(ensure(C.a_run_cnt, (size_t)nreg * 4 + 8));
    RET(ensure(C.a_run_off, (size_t)nreg * 8));
    RET(ensure(C.a_run_lo, (size_t)nreg * 8));
    RET(ensure(C.a_run_hi, (size_t)nreg * 8));
    {
        int* d_nruns = (int*)(C.a_run_cnt.as<char>() + (size_t)nreg * 4);
        size_t tb = 0;
        CK(cub::DeviceRunLengthEncode::Encode(nullptr, tb, aa.reg_key, C.a_run_key.as<unsigned long long>(),
                                              C.a_run_cnt.as<int>(), d_nruns, (int)nreg, st));
        RET(ensure(C.cub_tmp, tb));
        CK(cub::DeviceRunLengthEncode::Encode(C.cub_tmp.p, tb, aa.reg_key, C.a_run_key.as<unsigned long long>(),
                                              C.a_run_cnt.as<int>(), d_nruns, (int)nreg, st));
        int nruns = 0;
        RET(read_dev(d_nruns, nruns, st));
        RET(excl_scan(C, C.a_run_cnt.as<int>(), C.a_run_off.as<long long>(), nruns, st));
        CK(launch_ann_runs(C.a_run_cnt.as<unsigned>(), C.a_run_off.as<long long>(), nruns, C.a_run_lo.as<long long>(),
                           C.a_run_hi.as<long long>(), st));
        klaunch++;
        aa.nruns = nruns;
    }
    aa.run_key = C.a_run_key.as<unsigned long long>();
    aa.run_off = C.a_run_off.as<long long>();
    aa.run_cnt = C.a_run_cnt.as<int>();
    aa.run_lo = C.a_run_lo.as<long long>();
    aa.run_hi = C.a_run_hi.as<long long>();
    return PSIB_OK;
}

// Annihilation mode (src/cpsi.c:115-158): elements -> tets of both sides ->
// element pairs from a uniform cell grid -> tet pairs in the reference's order
// (e, e1 descending, t, t1), streamed in chunks -> one clip thread per tet pair
// -> records sorted by (voxel, tet pair) and summed into m.
int run_annihilation(Call& c)
{
    Ctx& C = *c.C;
    const psib_grid& g = *c.grid;
    const psib_mesh& m = *c.mesh;
    cudaStream_t st = c.st;
    const long long ne = m.nelem;
    const long long nvox = (long long)g.n[0] * g.n[1] * g.n[2];
    const GridDev gd = grid_dev(g);
    const MeshDev md = mesh_dev(m, g, c.pos, c.vel, c.mass, c.conn, c.reftol, nullptr);
    RET(ensure(C.small, S_WORDS * 8));
    unsigned long long* sm = C.small.as<unsigned long long>();
    CK(cudaMemsetAsync(sm, 0, S_WORDS * 8, st));
    long long klaunch = 0, launches = 0;
    float ms_tess = 0.f, ms_clip = 0.f, ms_final = 0.f;
    unsigned long long counts[3] = {0, 0, 0};
    long long ntp_total = 0;
    int nchunks = 0;
    auto fill_stats = [&](const unsigned long long* h) {
        if (!c.stats) return;
        psib_stats& s = *c.stats;
        s.elements_kept = (long long)h[S_TESS];
        s.tets = (long long)h[S_TESS + 1];
        s.tet_images = ntp_total;
        s.fragments = (long long)counts[0];
        s.frag_verts = (long long)counts[1];
        s.splits = (long long)counts[2];
        s.passes = 1;
        s.chunks = nchunks;
        s.ms_tess = ms_tess;
        s.ms_clip = ms_clip;
        s.ms_final = ms_final;
        s.clip_launches = launches;
        s.kernel_launches = klaunch + launches;
    };
    auto finish = [&]() -> int {
        unsigned long long h[S_WORDS];
        CK(cudaMemcpyAsync(h, sm, sizeof(h), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        RET(check_status(c, h));
        fill_stats(h);
        return PSIB_OK;
    };
    CK(cudaEventRecord(C.ev[2], st));

    // ---- elements: cull, side A and side B tets ----
    RET(ensure(C.a_cnt, (size_t)2 * (ne + 1) * sizeof(int)));
    RET(ensure(C.a_off, (size_t)2 * (ne + 1) * sizeof(long long)));
    RET(ensure(C.a_ebox, (size_t)(ne > 0 ? ne : 1) * 6 * sizeof(double)));
    int* cnt_a = C.a_cnt.as<int>();
    int* cnt_b = cnt_a + (ne + 1);
    long long* off_a = C.a_off.as<long long>();
    long long* off_b = off_a + (ne + 1);
    AnnTessArgs ta = {};
    ta.m = md;
    ta.g = gd;
    ta.max_lvl = c.maxlvl;
    ta.quad = m.elemtype == 27;
    ta.cnt_a = cnt_a;
    ta.cnt_b = cnt_b;
    ta.ebox = C.a_ebox.as<double>();
    ta.status = (unsigned*)&sm[S_STATUS];
    ta.counters = &sm[S_TESS];
    CK(launch_ann_tess(ta, false, st));
    klaunch++;
    CK(cudaMemsetAsync(cnt_a + ne, 0, sizeof(int), st));
    CK(cudaMemsetAsync(cnt_b + ne, 0, sizeof(int), st));
    RET(excl_scan(C, cnt_a, off_a, ne + 1, st));
    RET(excl_scan(C, cnt_b, off_b, ne + 1, st));
    long long na_tot = 0, nb_tot = 0;
    RET(read_dev(off_a + ne, na_tot, st));
    RET(read_dev(off_b + ne, nb_tot, st));
    {
        unsigned long long h[S_WORDS];
        CK(cudaMemcpy(h, sm, sizeof(h), cudaMemcpyDeviceToHost));
        RET(check_status(c, h));
    }
    if (na_tot >= (1ll << 31) || nb_tot >= (1ll << 31)) return fail(PSIB_ERR_OVERFLOW, "2^31 tets or more");
    if (na_tot == 0 || nb_tot == 0) return finish();
    RET(ensure(C.a_tets_a, (size_t)na_tot * TREC * sizeof(double)));
    RET(ensure(C.a_tets_b, (size_t)nb_tot * TREC * sizeof(double)));
    ta.off_a = off_a;
    ta.off_b = off_b;
    ta.tets_a = C.a_tets_a.as<double>();
    ta.tets_b = C.a_tets_b.as<double>();
    CK(launch_ann_tess(ta, true, st));
    klaunch++;

    // ---- the cell grid over the kept element boxes ----
    AnnArgs aa = {};
    aa.nelem = ne;
    aa.ebox = C.a_ebox.as<double>();
    aa.cnt_a = cnt_a;
    aa.cnt_b = cnt_b;
    aa.off_a = off_a;
    aa.off_b = off_b;
    aa.tets_a = ta.tets_a;
    aa.tets_b = ta.tets_b;
    aa.status = (unsigned*)&sm[S_STATUS];
    long long kept = 0;
    RET(build_cells(C, aa, st, klaunch, kept));
    if (kept == 0) return finish();
    const long long nreg = aa.nreg;

    // ---- element pairs, sorted (e ascending, e1 descending) ----
    RET(ensure(C.a_pair_cnt, (size_t)(nreg + 1) * sizeof(long long)));
    RET(ensure(C.a_pair_off, (size_t)(nreg + 1) * sizeof(long long)));
    aa.pair_cnt = C.a_pair_cnt.as<long long>();
    CK(launch_ann_pairs(aa, false, st));
    CK(cudaMemsetAsync(aa.pair_cnt + nreg, 0, sizeof(long long), st));
    RET(excl_scan(C, aa.pair_cnt, C.a_pair_off.as<long long>(), nreg + 1, st));
    long long npair = 0;
    RET(read_dev(C.a_pair_off.as<long long>() + nreg, npair, st));
    if (npair >= (1ll << 31)) return fail(PSIB_ERR_OVERFLOW, "too many element pairs (%lld)", npair);
    RET(ensure(C.a_pair_key, (size_t)(npair > 0 ? npair : 1) * 8));
    RET(ensure(C.a_pair_key_s, (size_t)(npair > 0 ? npair : 1) * 8));
    aa.pair_off = C.a_pair_off.as<long long>();
    aa.pair_key = C.a_pair_key.as<unsigned long long>();
    CK(launch_ann_pairs(aa, true, st));
    klaunch += 2;
    {
        size_t tb = 0;
        const int kb = 32 + bits_for((unsigned long long)ne);
        CK(cub::DeviceRadixSort::SortKeys(nullptr, tb, aa.pair_key, C.a_pair_key_s.as<unsigned long long>(), (int)npair,
                                          0, kb, st));
        RET(ensure(C.cub_tmp, tb));
        CK(cub::DeviceRadixSort::SortKeys(C.cub_tmp.p, tb, aa.pair_key, C.a_pair_key_s.as<unsigned long long>(),
                                          (int)npair, 0, kb, st));
    }
    aa.pair_key = C.a_pair_key_s.as<unsigned long long>();
    aa.npair = npair;

    // ---- tet-pair slots: side-A tets of each element pair; tet pairs per slot ----
    RET(ensure(C.a_na, (size_t)(npair + 1) * sizeof(long long)));
    RET(ensure(C.a_aoff, (size_t)(npair + 1) * sizeof(long long)));
    CK(launch_ann_pair_sides(aa, C.a_na.as<long long>(), st));
    CK(cudaMemsetAsync(C.a_na.as<long long>() + npair, 0, sizeof(long long), st));
    RET(excl_scan(C, C.a_na.as<long long>(), C.a_aoff.as<long long>(), npair + 1, st));
    long long nslot = 0;
    RET(read_dev(C.a_aoff.as<long long>() + npair, nslot, st));
    if (nslot >= (1ll << 31)) return fail(PSIB_ERR_OVERFLOW, "too many tet slots (%lld)", nslot);
    aa.aoff = C.a_aoff.as<long long>();
    aa.nslot = nslot;
    RET(ensure(C.a_tp_cnt, (size_t)(nslot + 1) * sizeof(long long)));
    RET(ensure(C.a_tp_excl, (size_t)(nslot + 1) * sizeof(long long)));
    aa.tp_cnt = C.a_tp_cnt.as<long long>();
    aa.slot0 = 0;
    aa.slot1 = nslot;
    CK(launch_ann_tpairs(aa, false, st));
    CK(cudaMemsetAsync(aa.tp_cnt + nslot, 0, sizeof(long long), st));
    RET(excl_scan(C, aa.tp_cnt, C.a_tp_excl.as<long long>(), nslot + 1, st));
    RET(read_dev(C.a_tp_excl.as<long long>() + nslot, ntp_total, st));
    aa.tp_excl = C.a_tp_excl.as<long long>();
    klaunch += 3;
    CK(cudaEventRecord(C.ev[3], st));
    CK(cudaEventSynchronize(C.ev[3]));
    CK(cudaEventElapsedTime(&ms_tess, C.ev[2], C.ev[3]));
    if (ntp_total == 0) return finish();

    // ---- chunks of about `budget` tet pairs, on slot boundaries ----
    const long long budget = std::max<long long>(env_ll("PSIB_ANN_BUDGET", 1ll << 24), 1);
    const int nb = (int)std::min<long long>((ntp_total + budget - 1) / budget, 1 << 20);
    RET(ensure(C.a_bounds, (size_t)(nb + 1) * sizeof(long long)));
    CK(launch_ann_chunk_bounds(aa.tp_excl, nslot, budget, nb, C.a_bounds.as<long long>(), st));
    std::vector<long long> bnd(nb + 1), boff(nb + 1);
    CK(cudaMemcpyAsync(bnd.data(), C.a_bounds.p, (nb + 1) * sizeof(long long), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int k = 0; k <= nb; ++k)
        CK(cudaMemcpyAsync(&boff[k], aa.tp_excl + bnd[k], sizeof(long long), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    long long cap = 1;
    for (int k = 0; k < nb; ++k) cap = std::max(cap, boff[k + 1] - boff[k]);
    if (cap >= (1ll << 31)) return fail(PSIB_ERR_OVERFLOW, "a chunk of %lld tet pairs is too large", cap);
    RET(ensure(C.a_tpairs, (size_t)cap * sizeof(int2)));
    RET(ensure(C.a_deep, (size_t)cap * sizeof(int)));
    RET(ensure(C.a_tp_key, (size_t)cap * sizeof(uint16_t)));
    RET(ensure(C.a_tp_key_s, (size_t)cap * sizeof(uint16_t)));
    RET(ensure(C.a_ord_in, (size_t)cap * sizeof(int)));
    RET(ensure(C.a_ord, (size_t)cap * sizeof(int)));
    aa.tpairs = C.a_tpairs.as<int2>();
    aa.tp_key = C.a_tp_key.as<uint16_t>();
    aa.g = gd;

    const int clip_block = 128, big_block = 64;
    const int clip_grid = C.num_sms * ann_blocks_per_sm(false, clip_block);
    RET(ensure(C.scratch, ann_scratch_bytes(false) * (size_t)clip_grid * clip_block));
    const int vbits = bits_for((unsigned long long)nvox);
    if (c.fields_ready) CK(cudaStreamWaitEvent(st, c.fields_ready, 0));
    for (int k = 0; k < nb; ++k) {
        const long long ntp = boff[k + 1] - boff[k];
        if (ntp == 0) continue;
        nchunks++;
        CK(cudaEventRecord(C.ev[4], st));
        aa.slot0 = bnd[k];
        aa.slot1 = bnd[k + 1];
        aa.tp_base = boff[k];
        CK(launch_ann_tpairs(aa, true, st));
        // the clip's order: larger walks first (k_ann_tpairs' keys)
        k_iota<<<C.num_sms * 8, 256, 0, st>>>(C.a_ord_in.as<int>(), ntp);
        CK(cudaGetLastError());
        {
            size_t tb = 0;
            CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, aa.tp_key, C.a_tp_key_s.as<uint16_t>(),
                                               C.a_ord_in.as<int>(), C.a_ord.as<int>(), (int)ntp, 0, 16, st));
            RET(ensure(C.cub_tmp, tb));
            CK(cub::DeviceRadixSort::SortPairs(C.cub_tmp.p, tb, aa.tp_key, C.a_tp_key_s.as<uint16_t>(),
                                               C.a_ord_in.as<int>(), C.a_ord.as<int>(), (int)ntp, 0, 16, st));
        }
        klaunch += 2;
        const int ibits = bits_for((unsigned long long)ntp);
        if (ibits + vbits > 64) return fail(PSIB_ERR_OVERFLOW, "grid and chunk too large for a 64-bit record key");
        AnnClipArgs ca = {};
        ca.tpairs = aa.tpairs;
        ca.tets_a = ta.tets_a;
        ca.tets_b = ta.tets_b;
        ca.g = gd;
        ca.deep = C.a_deep.as<int>();
        ca.ndeep = &sm[S_NDEEP];
        ca.rec_n = &sm[S_RECN];
        ca.rec_ibits = ibits;
        ca.status = (unsigned*)&sm[S_STATUS];
        ca.counters = &sm[S_CNT];
        unsigned long long nrec = 0;
        for (int attempt = 0;; ++attempt) {
            const unsigned long long want = (unsigned long long)std::max<long long>(ntp * 4, 1 << 16);
            RET(ensure(C.rkey, std::max<size_t>(C.rkey.n, want * 8)));
            RET(ensure(C.rmom, std::max<size_t>(C.rmom.n, C.rkey.n)));
            ca.rec_key = C.rkey.as<unsigned long long>();
            ca.rec_val = C.rmom.as<double>();
            ca.rec_cap = std::min<unsigned long long>(C.rkey.n / 8, C.rmom.n / 8);
            CK(cudaMemsetAsync(&sm[S_RECN], 0, 16, st)); // records, deep list
            CK(cudaMemsetAsync(&sm[S_CNT], 0, 24, st));
            CK(cudaMemsetAsync(&sm[S_HEAD], 0, 16, st));
            ca.n = ntp;
            ca.list = C.a_ord.as<int>();
            ca.head = &sm[S_HEAD];
            ca.scratch = C.scratch.p;
            CK(launch_ann_clip(ca, false, clip_grid, clip_block, st));
            launches++;
            unsigned long long ndeep = 0;
            RET(read_dev(&sm[S_NDEEP], ndeep, st));
            if (ndeep > 0) {
                const int big_grid =
                    (int)std::min<long long>((long long)C.num_sms * ann_blocks_per_sm(true, big_block),
                                             ((long long)ndeep + big_block - 1) / big_block);
                RET(ensure(C.scratch_big, ann_scratch_bytes(true) * (size_t)big_grid * big_block));
                ca.n = (long long)ndeep;
                ca.list = C.a_deep.as<int>();
                ca.head = &sm[S_HEAD + 1];
                ca.scratch = C.scratch_big.p;
                CK(launch_ann_clip(ca, true, big_grid, big_block, st));
                launches++;
            }
            unsigned long long h[S_WORDS];
            CK(cudaMemcpyAsync(h, sm, sizeof(h), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            nrec = h[S_RECN];
            if (nrec > ca.rec_cap && attempt == 0) {
                RET(ensure(C.rkey, nrec * 8));
                RET(ensure(C.rmom, nrec * 8));
                unsigned clr = 0;
                CK(cudaMemcpy(&sm[S_STATUS], &clr, sizeof(clr), cudaMemcpyHostToDevice));
                continue;
            }
            RET(check_status(c, h));
            for (int w = 0; w < 3; ++w) counts[w] += h[S_CNT + w];
            break;
        }
        CK(cudaEventRecord(C.ev[5], st));
        if (nrec >= (1ull << 32)) return fail(PSIB_ERR_OVERFLOW, "too many fragments in one chunk");
        if (nrec > 0) {
            // ---- records sorted by (voxel, tet pair), each voxel's run summed in that order ----
            RET(ensure(C.rkey_sorted, nrec * 8));
            RET(ensure(C.rperm_in, nrec * 4));
            RET(ensure(C.rperm, nrec * 4));
            RET(ensure(C.rvox, nrec * 4));
            RET(ensure(C.ritem, nrec * 4));
            RET(ensure(C.rmom_sorted, nrec * 8));
            const long long maxruns = std::min<long long>((long long)nrec, nvox);
            RET(ensure(C.run_vox, (size_t)maxruns * 4));
            RET(ensure(C.run_cnt, (size_t)maxruns * 4 + 8));
            RET(ensure(C.run_off, (size_t)maxruns * 8));
            k_iota<<<C.num_sms * 8, 256, 0, st>>>(C.rperm_in.as<unsigned>(), (long long)nrec);
            CK(cudaGetLastError());
            size_t tb = 0;
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
            ga.nmom = 1;
            ga.ibits = ibits;
            ga.vox = C.rvox.as<unsigned>();
            ga.item = C.ritem.as<unsigned>();
            ga.mom_sorted = C.rmom_sorted.as<double>();
            CK(launch_gather_records(ga, st));
            int* d_nruns = (int*)(C.run_cnt.as<char>() + (size_t)maxruns * 4);
            tb = 0;
            CK(cub::DeviceRunLengthEncode::Encode(nullptr, tb, C.rvox.as<unsigned>(), C.run_vox.as<unsigned>(),
                                                  C.run_cnt.as<int>(), d_nruns, (int)nrec, st));
            RET(ensure(C.cub_tmp, tb));
            CK(cub::DeviceRunLengthEncode::Encode(C.cub_tmp.p, tb, C.rvox.as<unsigned>(), C.run_vox.as<unsigned>(),
                                                  C.run_cnt.as<int>(), d_nruns, (int)nrec, st));
            int nruns = 0;
            RET(read_dev(d_nruns, nruns, st));
            RET(excl_scan(C, C.run_cnt.as<int>(), C.run_off.as<long long>(), nruns, st));
            ApplyArgs ap = {};
            ap.run_vox = C.run_vox.as<unsigned>();
            ap.run_cnt = C.run_cnt.as<int>();
            ap.run_off = C.run_off.as<long long>();
            ap.nruns = nruns;
            ap.mom = C.rmom_sorted.as<double>();
            ap.nmom = 1;
            ap.M = c.F[0];
            CK(launch_ann_apply(ap, st));
            klaunch += 3;
        }
        CK(cudaEventRecord(C.ev[6], st));
        CK(cudaEventSynchronize(C.ev[6]));
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, C.ev[4], C.ev[5]));
        ms_clip += t;
        CK(cudaEventElapsedTime(&t, C.ev[5], C.ev[6]));
        ms_final += t;
    }
    return finish();
}

} // namespace host
} // namespace psib
