// state_io.cu — binary checkpoint / resume of a solver's dynamic state and
// the multi-component station files.
//
// The reference keeps no restartable state: its only outputs are text slices
// and volumes of txx (OPT/ElasticWaveEquation.cu:843-948) and one txx station
// file (OPT/ElasticWaveEquation.cu:950-960).  A checkpoint here holds what a
// time step reads and writes besides the static inputs: the 9 wavefields, the
// 24 PML split fields, the traces and the next step index.  Medium, source,
// receivers and wavelet are the caller's inputs and are set again before a
// resume.
//
// Format (little-endian), version 2:
//   header, 128 bytes: see CkptHeader below;
//   payload: 9 fields of nx*ny*nz float32 (x fastest, in SGFD_VX..SGFD_TYZ
//   order), then the 24 PML splits as the library holds them: PML cells in
//   sgfd's pml_index order, in blocks of 32 cells, each block 24 rows of 32
//   float32 (split k of cell c at (c / 32) * 768 + 32 k + c % 32; the last
//   block zero-padded), then the traces, nt*nrec float32 time-major.
//   (Version 1 stored the splits split-major, 24 arrays of npml values.)
// The header's checksum covers the payload (4-lane FNV-1a over 64-bit words).
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "solver.h"

using namespace sgfd;

namespace {

constexpr char kMagic[8] = {'S', 'G', 'F', 'D', 'C', 'K', 'P', '1'};
constexpr uint32_t kVersion = 2;
constexpr size_t kStage = size_t(32) << 20;   // pinned staging chunk

struct CkptHeader {
    char magic[8];
    uint32_t version;
    uint32_t header_bytes;
    int32_t nx, ny, nz, pml;
    int32_t nrec, nt, it_next;
    int32_t quirks, damping, arith;
    float dt, dx, dy, dz;
    int64_t npml;
    uint64_t payload_bytes;
    uint64_t checksum;
    int8_t scale_e[9];   // 16-bit storage: exponents of the field scales (0 for FP32)
    uint8_t storage;     // sgfd_storage of the payload's values
    uint8_t pad0[2];
    int32_t nz_total, z_offset;   // z-slab: the whole model's GRID nz and the slab's offset (0, 0: whole model)
    uint8_t pad[128 - 8 - 8 - 16 - 12 - 12 - 16 - 24 - 10 - 2 - 8];
};
static_assert(sizeof(CkptHeader) == 128, "checkpoint header is 128 bytes");

// 4 independent FNV-1a lanes over 64-bit words (so the multiply chains
// overlap), folded at the end; a tail shorter than 32 bytes is hashed
// byte-wise into lane 0.
struct Checksum {
    uint64_t lane[4] = {0xcbf29ce484222325ull, 0x84222325cbf29ce4ull, 0x9ce484222325cbf2ull, 0x2325cbf29ce48422ull};
    std::vector<unsigned char> carry;   // bytes not yet forming a 32-byte block
    static constexpr uint64_t kPrime = 0x100000001b3ull;

    void block(const unsigned char *p, size_t n) {   // n multiple of 32
        for (size_t i = 0; i < n; i += 32) {
            uint64_t w[4];
            std::memcpy(w, p + i, 32);
            for (int k = 0; k < 4; ++k) lane[k] = (lane[k] ^ w[k]) * kPrime;
        }
    }
    void add(const void *data, size_t n) {
        const unsigned char *p = static_cast<const unsigned char *>(data);
        if (!carry.empty()) {
            const size_t take = std::min(n, 32 - carry.size());
            carry.insert(carry.end(), p, p + take);
            p += take; n -= take;
            if (carry.size() == 32) { block(carry.data(), 32); carry.clear(); }
        }
        const size_t whole = n / 32 * 32;
        block(p, whole);
        carry.insert(carry.end(), p + whole, p + n);
    }
    uint64_t value() const {
        uint64_t h = lane[0];
        for (unsigned char c : carry) h = (h ^ c) * kPrime;
        for (int k = 1; k < 4; ++k) h = (h ^ lane[k]) * kPrime;
        return h;
    }
};

// Byte sink / source over a caller's buffer or a FILE*.
struct Stream {
    unsigned char *mem = nullptr;
    const unsigned char *cmem = nullptr;
    size_t cap = 0, pos = 0;
    FILE *fp = nullptr;
    bool write(const void *p, size_t n) {
        if (fp) return std::fwrite(p, 1, n, fp) == n;
        if (pos + n > cap) return false;
        std::memcpy(mem + pos, p, n);
        pos += n;
        return true;
    }
    bool read(void *p, size_t n) {
        if (fp) return std::fread(p, 1, n, fp) == n;
        if (pos + n > cap) return false;
        std::memcpy(p, cmem + pos, n);
        pos += n;
        return true;
    }
};

struct PinnedDeleter {
    void operator()(void *p) const { cudaFreeHost(p); }
};

// One device region of the payload: `rows` rows of `row_bytes`, `pitch`
// bytes apart on the device, contiguous in the checkpoint.
struct Region {
    char *dev;
    size_t pitch, row_bytes, rows;
};

std::vector<Region> payload_regions(sgfd_solver *h) {
    const Model &m = h->m;
    std::vector<Region> r;
    for (int k = 0; k < SGFD_NFIELDS; ++k)
        r.push_back({reinterpret_cast<char *>(m.f[k]), (size_t)m.px * 4, (size_t)m.nx * 4, (size_t)m.ny * m.nz});
    if (m.npml > 0) {
        const size_t b = (size_t)split_elems(m.npml) * 4;
        r.push_back({reinterpret_cast<char *>(h->split), b, b, 1});
    }
    if (h->traces && h->sr.nrec > 0) {
        const size_t b = (size_t)h->sr.nrec * h->sr.nt * 4;
        r.push_back({reinterpret_cast<char *>(h->traces), b, b, 1});
    }
    return r;
}

uint64_t payload_bytes(sgfd_solver *h) {
    uint64_t n = 0;
    for (const Region &g : payload_regions(h)) n += (uint64_t)g.row_bytes * g.rows;
    return n;
}

void fill_header(sgfd_solver *h, int32_t it_next, CkptHeader *hd) {
    std::memset(hd, 0, sizeof *hd);
    std::memcpy(hd->magic, kMagic, 8);
    hd->version = kVersion;
    hd->header_bytes = sizeof *hd;
    const sgfd_config &c = h->cfg;
    hd->nx = c.nx; hd->ny = c.ny; hd->nz = c.nz; hd->pml = c.pml;
    hd->nrec = h->sr.nrec; hd->nt = h->sr.nt; hd->it_next = it_next;
    hd->quirks = c.quirks; hd->damping = c.damping; hd->arith = c.arith;
    hd->dt = c.dt; hd->dx = c.dx; hd->dy = c.dy; hd->dz = c.dz;
    hd->npml = h->m.npml;
    hd->payload_bytes = payload_bytes(h);
    hd->storage = (uint8_t)h->storage;
    hd->nz_total = c.nz_total;
    hd->z_offset = c.z_offset;
}

// Regions move through the staging chunk as whole rows where a row fits
// (fields) and as consecutive pieces of one row where it does not (the split
// array and the traces are single contiguous rows); either way the payload
// bytes come out in region order.
int save_state(sgfd_solver *h, int32_t it_next, Stream &out) {
    int r = check_handle(h);
    if (r) return r;
    if (it_next < 0) return fail(h, SGFD_ERR_INVALID, "negative step index");
    CkptHeader hd;
    fill_header(h, it_next, &hd);
    int e[9];
    r = get_scale_exponents(h, e);
    if (r == SGFD_OK) r = sync_views(h);   // 16-bit storage: the payload holds the read-back values
    if (r) return r;
    for (int g = 0; g < 9; ++g) hd.scale_e[g] = (int8_t)e[g];
    const long hdr_pos = out.fp ? std::ftell(out.fp) : (long)out.pos;
    if (!out.write(&hd, sizeof hd)) return fail(h, SGFD_ERR_INVALID, "checkpoint buffer too small or write failed");
    void *raw = nullptr;
    SG_CUDA(h, cudaMallocHost(&raw, kStage), "checkpoint staging buffer");
    std::unique_ptr<void, PinnedDeleter> stage(raw);
    unsigned char *st = static_cast<unsigned char *>(raw);
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "checkpoint: finish queued steps");
    r = check_device_error(h);
    if (r) return r;
    Checksum ck;
    for (const Region &g : payload_regions(h)) {
        const size_t rows_per = g.row_bytes > kStage ? 1 : kStage / g.row_bytes;
        for (size_t r0 = 0; r0 < g.rows; r0 += rows_per) {
            const size_t nr = std::min(rows_per, g.rows - r0);
            for (size_t off = 0; off < g.row_bytes; off += kStage) {   // pieces of a row longer than the chunk
                const size_t piece = std::min(kStage, g.row_bytes - off);
                const char *src = g.dev + r0 * g.pitch + off;
                SG_CUDA(h, nr == 1 ? cudaMemcpyAsync(st, src, piece, cudaMemcpyDeviceToHost, h->stream)
                                   : cudaMemcpy2DAsync(st, piece, src, g.pitch, piece, nr, cudaMemcpyDeviceToHost,
                                                       h->stream), "checkpoint download");
                SG_CUDA(h, cudaStreamSynchronize(h->stream), "checkpoint download");
                ck.add(st, piece * nr);
                if (!out.write(st, piece * nr)) return fail(h, SGFD_ERR_INVALID, "checkpoint write failed");
            }
        }
    }
    hd.checksum = ck.value();
    if (out.fp) {
        const long end = std::ftell(out.fp);
        if (std::fseek(out.fp, hdr_pos, SEEK_SET) != 0 || std::fwrite(&hd, sizeof hd, 1, out.fp) != 1 ||
            std::fseek(out.fp, end, SEEK_SET) != 0)
            return fail(h, SGFD_ERR_INVALID, "checkpoint header write failed");
    } else {
        std::memcpy(out.mem + hdr_pos, &hd, sizeof hd);
    }
    return SGFD_OK;
}

int load_state(sgfd_solver *h, Stream &in, int32_t *it_next) {
    int r = check_handle(h);
    if (r) return r;
    CkptHeader hd, want;
    if (!in.read(&hd, sizeof hd)) return fail(h, SGFD_ERR_INVALID, "checkpoint shorter than its header");
    if (std::memcmp(hd.magic, kMagic, 8) != 0) return fail(h, SGFD_ERR_INVALID, "not an sgfd checkpoint");
    if (hd.version != kVersion || hd.header_bytes != sizeof hd)
        return fail(h, SGFD_ERR_UNSUPPORTED, "checkpoint version %u not supported", hd.version);
    fill_header(h, 0, &want);
    if (hd.nx != want.nx || hd.ny != want.ny || hd.nz != want.nz || hd.pml != want.pml || hd.npml != want.npml)
        return fail(h, SGFD_ERR_INVALID, "checkpoint grid %dx%dx%d pml %d does not match the solver's %dx%dx%d pml %d",
                    hd.nx, hd.ny, hd.nz, hd.pml, want.nx, want.ny, want.nz, want.pml);
    if (hd.nz_total != want.nz_total || hd.z_offset != want.z_offset)
        return fail(h, SGFD_ERR_INVALID, "checkpoint of the z-slab at plane %d of %d planes, the solver is at %d of %d",
                    hd.z_offset, hd.nz_total, want.z_offset, want.nz_total);
    if (hd.nrec != want.nrec || hd.nt != want.nt)
        return fail(h, SGFD_ERR_INVALID, "checkpoint holds %d receivers x %d steps, the solver %d x %d",
                    hd.nrec, hd.nt, want.nrec, want.nt);
    if (hd.quirks != want.quirks || hd.damping != want.damping || hd.dt != want.dt || hd.dx != want.dx ||
        hd.dy != want.dy || hd.dz != want.dz)
        return fail(h, SGFD_ERR_INVALID, "checkpoint physics (dt, cell sizes, damping, quirks) differ from the solver's");
    if (hd.payload_bytes != want.payload_bytes) return fail(h, SGFD_ERR_INVALID, "checkpoint payload size mismatch");
    if (hd.storage != want.storage)
        return fail(h, SGFD_ERR_INVALID, "checkpoint storage type %d differs from the solver's %d", hd.storage,
                    want.storage);
    void *raw = nullptr;
    SG_CUDA(h, cudaMallocHost(&raw, kStage), "checkpoint staging buffer");
    std::unique_ptr<void, PinnedDeleter> stage(raw);
    unsigned char *st = static_cast<unsigned char *>(raw);
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "checkpoint: finish queued steps");
    Checksum ck;
    bool short_read = false;
    for (const Region &g : payload_regions(h)) {
        const size_t rows_per = g.row_bytes > kStage ? 1 : kStage / g.row_bytes;
        for (size_t r0 = 0; r0 < g.rows && !short_read; r0 += rows_per) {
            const size_t nr = std::min(rows_per, g.rows - r0);
            for (size_t off = 0; off < g.row_bytes; off += kStage) {
                const size_t piece = std::min(kStage, g.row_bytes - off);
                if (!in.read(st, piece * nr)) { short_read = true; break; }
                ck.add(st, piece * nr);
                char *dst = g.dev + r0 * g.pitch + off;
                SG_CUDA(h, nr == 1 ? cudaMemcpyAsync(dst, st, piece, cudaMemcpyHostToDevice, h->stream)
                                   : cudaMemcpy2DAsync(dst, g.pitch, st, piece, piece, nr, cudaMemcpyHostToDevice,
                                                       h->stream), "checkpoint upload");
                SG_CUDA(h, cudaStreamSynchronize(h->stream), "checkpoint upload");
            }
        }
    }
    if (short_read || ck.value() != hd.checksum) {
        sgfd_reset(h);   // do not leave a half-loaded state behind
        return fail(h, SGFD_ERR_INVALID, short_read ? "checkpoint truncated; state reset to zero"
                                                    : "checkpoint checksum mismatch; state reset to zero");
    }
    if (h->storage != SGFD_STORE_F32) {   // back to 16-bit values under the saved scales
        int e[9];
        for (int g = 0; g < 9; ++g) e[g] = hd.scale_e[g];
        r = set_scale_exponents(h, e);
        if (r == SGFD_OK) r = sync_from_views(h);
        if (r) return r;
        SG_CUDA(h, cudaStreamSynchronize(h->stream), "checkpoint: 16-bit values");
    }
    if (it_next) *it_next = hd.it_next;
    return SGFD_OK;
}

const char *comp_name(int c) {
    static const char *names[SGFD_NFIELDS] = {"vx", "vy", "vz", "txx", "tyy", "tzz", "txy", "txz", "tyz"};
    return c >= 0 && c < SGFD_NFIELDS ? names[c] : "unknown";
}

}  // namespace

extern "C" {

int sgfd_checkpoint_bytes(sgfd_solver *h, int64_t *bytes) {
    int r = check_handle(h);
    if (r) return r;
    if (!bytes) return fail(h, SGFD_ERR_INVALID, "null output");
    *bytes = (int64_t)(sizeof(CkptHeader) + payload_bytes(h));
    return SGFD_OK;
}

int sgfd_checkpoint_save(sgfd_solver *h, int32_t it_next, void *buf, int64_t bytes) {
    if (!buf || bytes < 0) return fail(h, SGFD_ERR_INVALID, "null checkpoint buffer");
    Stream s;
    s.mem = static_cast<unsigned char *>(buf);
    s.cap = (size_t)bytes;
    return save_state(h, it_next, s);
}

int sgfd_checkpoint_load(sgfd_solver *h, const void *buf, int64_t bytes, int32_t *it_next) {
    if (!buf || bytes < 0) return fail(h, SGFD_ERR_INVALID, "null checkpoint buffer");
    Stream s;
    s.cmem = static_cast<const unsigned char *>(buf);
    s.cap = (size_t)bytes;
    return load_state(h, s, it_next);
}

int sgfd_checkpoint_write(sgfd_solver *h, int32_t it_next, const char *path) {
    if (!path) return fail(h, SGFD_ERR_INVALID, "null path");
    FILE *fp = std::fopen(path, "wb");
    if (!fp) return fail(h, SGFD_ERR_INVALID, "cannot open %s for writing", path);
    Stream s;
    s.fp = fp;
    int r = save_state(h, it_next, s);
    if (std::fclose(fp) != 0 && r == SGFD_OK) r = fail(h, SGFD_ERR_INVALID, "closing %s failed", path);
    return r;
}

int sgfd_checkpoint_read(sgfd_solver *h, const char *path, int32_t *it_next) {
    if (!path) return fail(h, SGFD_ERR_INVALID, "null path");
    FILE *fp = std::fopen(path, "rb");
    if (!fp) return fail(h, SGFD_ERR_INVALID, "cannot open %s", path);
    Stream s;
    s.fp = fp;
    int r = load_state(h, s, it_next);
    std::fclose(fp);
    return r;
}

int sgfd_write_stations(sgfd_solver *h, const char *prefix, int32_t nsteps, int32_t binary) {
    int r = check_handle(h);
    if (r) return r;
    if (!prefix) return fail(h, SGFD_ERR_INVALID, "null prefix");
    const int n = h->sr.nrec, nt = h->sr.nt;
    if (n == 0) return fail(h, SGFD_ERR_STATE, "no receivers set");
    if (nsteps < 0 || nsteps > nt) return fail(h, SGFD_ERR_INVALID, "nsteps %d outside [0, %d]", nsteps, nt);
    if (nsteps == 0) nsteps = nt;
    std::vector<float> tm((size_t)n * nt);
    SG_CUDA(h, cudaMemcpyAsync(tm.data(), h->traces, tm.size() * sizeof(float), cudaMemcpyDeviceToHost, h->stream),
            "trace download");
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "trace download");
    r = check_device_error(h);
    if (r) return r;
    const std::string pre(prefix);
    // receiver table: index, x, y, z, component, column within its component file
    FILE *fr = std::fopen((pre + "_receivers.txt").c_str(), "w");
    if (!fr) return fail(h, SGFD_ERR_INVALID, "cannot open %s_receivers.txt", prefix);
    std::fprintf(fr, "# receiver x y z component column\n");
    int col[SGFD_NFIELDS] = {0};
    std::vector<std::vector<int>> members(SGFD_NFIELDS);
    for (int q = 0; q < n; ++q) {
        const int4 &p = h->rec_host[q];
        std::fprintf(fr, "%d %d %d %d %s %d\n", q, p.x, p.y, p.z, comp_name(p.w), col[p.w]++);
        members[p.w].push_back(q);
    }
    std::fclose(fr);
    // one file per recorded component: nsteps lines x (its receivers) columns
    std::vector<float> row;
    for (int c = 0; c < SGFD_NFIELDS; ++c) {
        if (members[c].empty()) continue;
        const std::string base = pre + "_" + comp_name(c);
        FILE *ft = std::fopen((base + ".txt").c_str(), "w");
        FILE *fb = binary ? std::fopen((base + ".bin").c_str(), "wb") : nullptr;
        if (!ft || (binary && !fb)) {
            if (ft) std::fclose(ft);
            if (fb) std::fclose(fb);
            return fail(h, SGFD_ERR_INVALID, "cannot open %s output", base.c_str());
        }
        const int nc = (int)members[c].size();
        if (fb) {   // binary twin: int32 nsteps, int32 ncols, then float32 [nsteps][ncols]
            const int32_t dims[2] = {nsteps, nc};
            std::fwrite(dims, sizeof dims, 1, fb);
        }
        row.resize(nc);
        for (int it = 0; it < nsteps; ++it) {
            for (int k = 0; k < nc; ++k) {
                row[k] = tm[(size_t)it * n + members[c][k]];
                std::fprintf(ft, k ? " %g" : "%g", (double)row[k]);
            }
            std::fputc('\n', ft);
            if (fb) std::fwrite(row.data(), sizeof(float), nc, fb);
        }
        const bool bad = std::ferror(ft) || (fb && std::ferror(fb));
        std::fclose(ft);
        if (fb) std::fclose(fb);
        if (bad) return fail(h, SGFD_ERR_INVALID, "writing %s failed", base.c_str());
    }
    return SGFD_OK;
}

}  // extern "C"
