/*
 * loaders.cpp -- snapshot readers of the C ABI: a Gadget-2 (format 1) file
 * becomes the periodic trilinear mesh that PSI.Mesh(loader='gadget2' |
 * 'gevolution') builds in the reference (src/mesh.c:35-302, src/PSI.c:659-709).
 *
 * File layout (native byte order, every block framed by a 4-byte length
 * before and after it): a 256-byte header, then float32 positions (npart x 3),
 * float32 velocities (npart x 3) and particle IDs (int32 for Gadget-2, int64
 * for gevolution).  Only type-1 particles are read, npart = header.npart[1].
 * Particle p lands at row ID[p] of pos and vel; every element's mass is
 * header.mass[1] / npart; the box is [0, BoxSize]^3, periodic.
 *
 * Gadget-2 connectivity: the IDs are the row-major index of an n^3 lattice
 * (n = npart^(1/3)) and element e = n^2 i + n j + k joins the particles at the
 * corners (i+ii, j+jj, k+kk) mod n in the corner order 4 ii + 2 jj + kk.
 * gevolution numbers its particles in tiles of 4^3: the ID is 64 x (tile
 * index, i fastest) + the position inside the tile along a two-level Gray
 * code; element p is the cube of particle p and its 7 upper neighbours.
 *
 * Differences from the reference, all on files it would read out of bounds or
 * leave partly uninitialised: an ID outside [0, npart) or repeated, a particle
 * count that is not a cube (gevolution: a cube of a multiple of 4 per side),
 * and a block whose length marker disagrees with npart are errors here.
 *
 * The IDs are read first and the position and velocity blocks are then
 * streamed in chunks straight into their rows, so a load needs no float copy
 * of the particle data; the scatter of each chunk, the masses and the
 * connectivity are filled by up to 16 host threads.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "psi_b200.h"

namespace psib {
int report_error(int code, const char* msg);  // sets the message psib_last_error() returns
}

namespace {

constexpr long HEADER_BYTES = 256;
// byte offsets inside the header (npart[6] int32, mass[6] double, time, redshift,
// 2 int32 flags, npartTotal[6], 2 int32, BoxSize, ...)
constexpr long OFF_NPART1 = 4;
constexpr long OFF_MASS1 = 24 + 8;
constexpr long OFF_BOXSIZE = 128;

int fail(int code, const std::string& msg) { return psib::report_error(code, msg.c_str()); }

struct File {
    FILE* f = nullptr;
    explicit File(const char* name) : f(name ? std::fopen(name, "rb") : nullptr) {}
    ~File()
    {
        if (f) std::fclose(f);
    }
    bool read(void* dst, size_t bytes) { return std::fread(dst, 1, bytes, f) == bytes; }
    bool seek(long long off) { return fseeko(f, (off_t)off, SEEK_SET) == 0; }
};

struct Header {
    long long npart = 0;
    double mass1 = 0.0, box = 0.0;
};

bool read_header(File& fp, Header& h)
{
    unsigned char raw[4 + HEADER_BYTES + 4];
    if (!fp.read(raw, sizeof raw)) return false;
    const unsigned char* hd = raw + 4;
    int32_t n1;
    std::memcpy(&n1, hd + OFF_NPART1, 4);
    std::memcpy(&h.mass1, hd + OFF_MASS1, 8);
    std::memcpy(&h.box, hd + OFF_BOXSIZE, 8);
    h.npart = n1;
    return true;
}

// the 4-byte length marker of a data block, which must equal `want` modulo 2^32
// (writers store the byte count of a block of 4 GiB or more wrapped)
bool marker(File& fp, unsigned long long want)
{
    uint32_t m;
    return fp.read(&m, 4) && m == (uint32_t)want;
}

// integer cube root: the n with n^3 <= v < (n+1)^3
long long icbrt(long long v)
{
    long long n = (long long)std::llround(std::cbrt((double)v));
    while (n > 0 && n * n * n > v) --n;
    while ((n + 1) * (n + 1) * (n + 1) <= v) ++n;
    return n;
}

// 3-bit reflected Gray code and its inverse; bit 2 is the i axis, bit 0 the k axis
inline int gray(int n) { return n ^ (n >> 1); }
inline int gray_inv(int g) { return g ^ (g >> 1) ^ (g >> 2); }

// position (i,j,k) in 0..3 of the particle at slot s of a 4^3 tile: an outer Gray
// code over the 2^3 sub-cubes of side 2, an inner one inside each sub-cube
inline void tile_slot_to_cube(int s, int c[3])
{
    int o = gray(s >> 3), in = gray(s & 7);
    for (int a = 0; a < 3; ++a) c[a] = 2 * ((o >> (2 - a)) & 1) + ((in >> (2 - a)) & 1);
}

inline int tile_cube_to_slot(int i, int j, int k)
{
    int o = ((i >> 1) << 2) | ((j >> 1) << 1) | (k >> 1);
    int in = ((i & 1) << 2) | ((j & 1) << 1) | (k & 1);
    return 8 * gray_inv(o) + gray_inv(in);
}

// Run f(begin, end) over [0, n) in contiguous ranges on up to 16 host threads.
template <class F>
void parallel_for(long long n, F f)
{
    const long long hw = std::max(1u, std::thread::hardware_concurrency());
    const long long nt = std::min<long long>(std::min<long long>(hw, 16), std::max<long long>(1, n / 16384));
    if (nt <= 1) {
        f(0, n);
        return;
    }
    std::vector<std::thread> th;
    for (long long t = 0; t < nt; ++t) th.emplace_back(f, n * t / nt, n * (t + 1) / nt);
    for (auto& x : th) x.join();
}

template <typename ID>
int load(const char* filename, bool tiled, long long npart, double* pos, double* vel, double* mass, int* conn)
{
    psib::report_error(PSIB_OK, "");
    if (!filename || !pos || !vel || !mass || !conn) return fail(PSIB_ERR_ARG, "filename and all output arrays are required");
    File fp(filename);
    if (!fp.f) return fail(PSIB_ERR_ARG, std::string("cannot open ") + filename);
    Header h;
    if (!read_header(fp, h)) return fail(PSIB_ERR_ARG, "truncated header");
    if (h.npart != npart)
        return fail(PSIB_ERR_ARG, "the output arrays hold " + std::to_string(npart) + " particles, the file " +
                                      std::to_string(h.npart));
    if (npart < 0) return fail(PSIB_ERR_ARG, "negative particle count in the header");
    const long long n = icbrt(npart);
    if (n * n * n != npart)
        return fail(PSIB_ERR_ARG, std::to_string(npart) + " particles do not form a cubic lattice");
    if (tiled && n % 4 != 0)
        return fail(PSIB_ERR_ARG, "a gevolution lattice needs a side that is a multiple of 4, not " + std::to_string(n));

    const unsigned long long vec_bytes = 12ull * (unsigned long long)npart;
    const unsigned long long id_bytes = sizeof(ID) * (unsigned long long)npart;
    const long long pos_at = 4 + HEADER_BYTES + 4;
    const long long vel_at = pos_at + 8 + (long long)vec_bytes;
    const long long id_at = vel_at + 8 + (long long)vec_bytes;

    // the IDs: every one in [0, npart) and none twice
    std::vector<int32_t> row((size_t)npart);
    {
        if (!fp.seek(id_at) || !marker(fp, id_bytes)) return fail(PSIB_ERR_ARG, "bad particle ID block");
        std::vector<uint8_t> seen((size_t)npart, 0);
        std::vector<ID> buf(1 << 16);
        for (long long p0 = 0; p0 < npart; p0 += (long long)buf.size()) {
            size_t cnt = (size_t)std::min<long long>((long long)buf.size(), npart - p0);
            if (!fp.read(buf.data(), cnt * sizeof(ID))) return fail(PSIB_ERR_ARG, "truncated particle ID block");
            for (size_t q = 0; q < cnt; ++q) {
                long long id = (long long)buf[q];
                if (id < 0 || id >= npart)
                    return fail(PSIB_ERR_INDEX, "particle ID " + std::to_string(id) + " outside [0, " +
                                                    std::to_string(npart) + ")");
                if (seen[(size_t)id]) return fail(PSIB_ERR_INDEX, "particle ID " + std::to_string(id) + " repeated");
                seen[(size_t)id] = 1;
                row[(size_t)(p0 + (long long)q)] = (int32_t)id;
            }
        }
        if (!marker(fp, id_bytes)) return fail(PSIB_ERR_ARG, "bad particle ID block");
    }

    // positions and velocities, float32 widened to double, scattered to their rows (the
    // IDs are distinct, so the threads of a chunk write distinct rows)
    std::vector<float> buf(3u << 20);
    for (int blk = 0; blk < 2; ++blk) {
        double* dst = blk ? vel : pos;
        if (!fp.seek(blk ? vel_at : pos_at) || !marker(fp, vec_bytes))
            return fail(PSIB_ERR_ARG, blk ? "bad velocity block" : "bad position block");
        for (long long p0 = 0; p0 < npart; p0 += (long long)buf.size() / 3) {
            size_t cnt = (size_t)std::min<long long>((long long)buf.size() / 3, npart - p0);
            if (!fp.read(buf.data(), cnt * 12)) return fail(PSIB_ERR_ARG, "truncated particle block");
            parallel_for((long long)cnt, [&](long long b, long long e) {
                for (long long q = b; q < e; ++q) {
                    double* d = dst + 3 * (size_t)row[(size_t)(p0 + q)];
                    d[0] = buf[3 * q];
                    d[1] = buf[3 * q + 1];
                    d[2] = buf[3 * q + 2];
                }
            });
        }
        if (!marker(fp, vec_bytes)) return fail(PSIB_ERR_ARG, blk ? "bad velocity block" : "bad position block");
    }

    const double m = h.mass1 / (double)npart;
    parallel_for(npart, [&](long long b, long long e) {
        for (long long i = b; i < e; ++i) mass[i] = m;
    });

    if (!tiled) {
        // element (i, j, k) joins the lattice points (i + ii, j + jj, k + kk) mod n
        const long long n2 = n * n;
        parallel_for(n, [&](long long i0, long long i1) {
            for (long long i = i0; i < i1; ++i) {
                const long long a[2] = {n2 * i, n2 * (i + 1 == n ? 0 : i + 1)};
                for (long long j = 0; j < n; ++j) {
                    const long long b[2] = {n * j, n * (j + 1 == n ? 0 : j + 1)};
                    int* c = conn + 8 * (n2 * i + n * j);
                    for (long long k = 0; k < n; ++k, c += 8) {
                        const long long kk[2] = {k, k + 1 == n ? 0 : k + 1};
                        for (int v = 0; v < 8; ++v) c[v] = (int)(a[v >> 2] + b[(v >> 1) & 1] + kk[v & 1]);
                    }
                }
            }
        });
    } else {
        // per tile: the flat index of its 8 upper neighbour tiles; per slot: its cube position;
        // per position in the 5^3 block of a slot and its upper neighbours: the slot inside the tile
        const long long tn = n / 4;
        int cube[64][3];
        for (int sl = 0; sl < 64; ++sl) tile_slot_to_cube(sl, cube[sl]);
        parallel_for(tn * tn * tn, [&](long long t0, long long t1) {
            for (long long t = t0; t < t1; ++t) {
                const long long ti = t % tn, tj = (t / tn) % tn, tk = t / (tn * tn);
                const long long tip = ti + 1 == tn ? 0 : ti + 1, tjp = tj + 1 == tn ? 0 : tj + 1,
                                tkp = tk + 1 == tn ? 0 : tk + 1;
                long long nbt[8]; // neighbour tile (di, dj, dk) at 4 di + 2 dj + dk
                for (int d = 0; d < 8; ++d)
                    nbt[d] = ((d >> 2) ? tip : ti) + tn * (((d >> 1) & 1) ? tjp : tj) + tn * tn * ((d & 1) ? tkp : tk);
                for (int sl = 0; sl < 64; ++sl) {
                    int* c = conn + 8 * (64 * t + sl);
                    for (int v = 0; v < 8; ++v) {
                        int q[3], d = 0;
                        for (int ax = 0; ax < 3; ++ax) {
                            q[ax] = cube[sl][ax] + ((v >> (2 - ax)) & 1);
                            d |= (q[ax] >> 2) << (2 - ax);
                            q[ax] &= 3;
                        }
                        c[v] = (int)(64 * nbt[d] + tile_cube_to_slot(q[0], q[1], q[2]));
                    }
                }
            }
        });
    }
    return PSIB_OK;
}

}  // namespace

extern "C" {

int psib_peek_gadget2(const char* filename, long long* npart, double* box_size)
{
    psib::report_error(PSIB_OK, "");
    if (!filename) return fail(PSIB_ERR_ARG, "filename is required");
    File fp(filename);
    if (!fp.f) return fail(PSIB_ERR_ARG, std::string("cannot open ") + filename);
    Header h;
    if (!read_header(fp, h)) return fail(PSIB_ERR_ARG, "truncated header");
    if (npart) *npart = h.npart;
    if (box_size) *box_size = h.box;
    return PSIB_OK;
}

int psib_load_gadget2(const char* filename, long long npart, double* pos, double* vel, double* mass, int* connectivity)
{
    return load<int32_t>(filename, false, npart, pos, vel, mass, connectivity);
}

int psib_load_gevolution(const char* filename, long long npart, double* pos, double* vel, double* mass,
                         int* connectivity)
{
    return load<int64_t>(filename, true, npart, pos, vel, mass, connectivity);
}

}  // extern "C"
