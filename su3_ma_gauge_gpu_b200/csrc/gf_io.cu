// gf_io.cu -- gauge-field files <-> the GpuPattern device layout, transcoded on the GPU.
//
// Formats (the reference's LinkFile and app readers):
//  PLAIN       the StandardPattern array, unique index c + 2*(j + 3*(i + 3*(mu + 4*l))) with the
//              lexicographic site l = ((t*Nx + x)*Ny + y)*Nz + z (access_pattern/StandardPattern.hxx:53-56,
//              lattice/LinkFile.hxx:83-167), no header;
//  HEADERONLY  an opaque header of (file size - array size) bytes, then PLAIN; written back as read
//              (lattice/filetypes/FileHeaderOnly.hxx:72-103);
//  VOGT        short ndim, short nc, short extents[ndim], short sizeof(real), then PLAIN
//              (lattice/filetypes/FileVogt.hxx:60-108);
//  ILDG        a LIME container whose "ildg-binary-data" record holds big-endian doubles in the order
//              ((((t*Nz + z)*Ny + y)*Nx + x)*4 + mu_f)*18 + 6*i + 2*j + c, file direction
//              mu_f = (x, y, z, t) -> mu = mu_f + 1 mod 4 (apps/ildg.cpp:26-97); on writing, the other
//              records of a template file are copied and "xlf-info" gets " SA steps N" appended
//              (apps/ildg.cpp:99-238);
//  QCDSTAG     raw native doubles in the order ((mu*Nt + t)*Nz + z)*Ny + y)*Nx + x)*18 + 6*i + 2*j + c;
//              the reference stores the file direction unchanged (apps/qcdstag.cpp:17-67).
// The file payload is read into pinned host memory, copied to the GPU once and transcoded there by
// one thread per link (byte order, element type, site order and direction permutation in one pass);
// the reference does the same element by element on the host through getIndexByUnique.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "gf_host.hpp"
#include "gf_kernels.cuh"

namespace gfb {

enum FileOrder : int { ORD_STANDARD = 0, ORD_ILDG = 1, ORD_QCDSTAG = 2 };

__device__ __forceinline__ double bswap_f64(double v)
{
    unsigned long long u = __double_as_longlong(v);
    u = ((u & 0x00000000FFFFFFFFull) << 32) | ((u & 0xFFFFFFFF00000000ull) >> 32);
    u = ((u & 0x0000FFFF0000FFFFull) << 16) | ((u & 0xFFFF0000FFFF0000ull) >> 16);
    u = ((u & 0x00FF00FF00FF00FFull) << 8) | ((u & 0xFF00FF00FF00FF00ull) >> 8);
    return __longlong_as_double((long long)u);
}

// file element offset of link (coords c, internal direction mu) and the internal <-> file direction
__device__ __forceinline__ int64_t file_link_offset(const Geom &g, const int32_t c[4], int mu, int order)
{
    const int64_t Nt = g.n[0], Nx = g.n[1], Ny = g.n[2], Nz = g.n[3];
    if (order == ORD_STANDARD) {
        const int64_t l = ((c[0] * Nx + c[1]) * Ny + c[2]) * Nz + c[3];
        return (l * 4 + mu) * 18;
    }
    const int64_t lf = ((c[0] * Nz + c[3]) * Ny + c[2]) * Nx + c[1];  // x fastest
    if (order == ORD_ILDG) {
        const int muf = (mu + 3) & 3;  // internal mu = file mu + 1 (mod 4)
        return (lf * 4 + muf) * 18;
    }
    return ((int64_t)mu * Nt * Nx * Ny * Nz + lf) * 18;  // QCDSTAG: file direction kept
}

// Memory side: GpuPattern (GF_LAYOUT_GPU, access_pattern/GpuPattern.hxx:53-56) or
// GpuPatternTimeslice (GF_LAYOUT_TIMESLICE, access_pattern/GpuPatternTimeslice.hxx:57-62: slice t
// is the GpuPattern array of the {1, Nx, Ny, Nz} lattice, spatial parity, at offset t * 72 Vs).
// Returns the offset of real 0 of link (coords c, mu) and the stride between its 18 reals.
__device__ __forceinline__ int64_t memory_link_offset(const Geom &g, const Geom &gs, const int32_t c[4], int mu,
                                                      int64_t s, int layout, int64_t &stride)
{
    if (layout == GF_LAYOUT_GPU) {
        stride = g.V;
        return (int64_t)mu * 18 * g.V + s;
    }
    const int32_t cs[4] = {0, c[1], c[2], c[3]};
    stride = gs.V;
    return (int64_t)c[0] * 72 * gs.V + (int64_t)mu * 18 * gs.V + site_index(gs, cs);
}

// one thread per link (s, mu): file buffer -> memory layout (all 18 reals)
template <typename Rf, typename R>
__global__ void __launch_bounds__(256) k_file_to_gpu(const Rf *file, Geom g, Geom gs, int order, int swap,
                                                     int layout, R *U)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 4 * g.V) return;
    const int mu = (int)(idx / g.V);
    const int64_t s = idx - mu * g.V;
    const int parity = s >= g.Vh;
    int32_t c[4];
    site_coords(g, s - (parity ? g.Vh : 0), parity, c);
    const Rf *src = file + file_link_offset(g, c, mu, order);
    int64_t stride;
    R *dst = U + memory_link_offset(g, gs, c, mu, s, layout, stride);
#pragma unroll
    for (int k = 0; k < 18; k++) {
        double v = (double)src[k];
        if (sizeof(Rf) == 8 && swap) v = bswap_f64(v);
        dst[k * stride] = (R)v;
    }
}

template <typename R, typename Rf>
__global__ void __launch_bounds__(256) k_gpu_to_file(const R *U, Geom g, Geom gs, int order, int swap, int layout,
                                                     Rf *file)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 4 * g.V) return;
    const int mu = (int)(idx / g.V);
    const int64_t s = idx - mu * g.V;
    const int parity = s >= g.Vh;
    int32_t c[4];
    site_coords(g, s - (parity ? g.Vh : 0), parity, c);
    Rf *dst = file + file_link_offset(g, c, mu, order);
    int64_t stride;
    const R *src = U + memory_link_offset(g, gs, c, mu, s, layout, stride);
#pragma unroll
    for (int k = 0; k < 18; k++) {
        double v = (double)src[k * stride];
        if (sizeof(Rf) == 8 && swap) v = bswap_f64(v);
        dst[k] = (Rf)v;
    }
}

// ---- LIME container (SciDAC LIME record format) -------------------------------------------------
// A record is a 144-byte header -- magic 0x456789ab, version, flags (bit 15 message begin,
// bit 14 message end), 64-bit data length, 128-byte type string, all big-endian -- followed by
// the data, padded with zeros to a multiple of 8 bytes.
struct LimeRecord {
    std::string type;
    bool mb = false, me = false;
    std::vector<char> data;  // for the binary record: only its offset/length are kept
    long long offset = 0, length = 0;
};

static uint64_t be64(const unsigned char *p)
{
    uint64_t v = 0;
    for (int i = 0; i < 8; i++) v = (v << 8) | p[i];
    return v;
}

static void put_be(unsigned char *p, uint64_t v, int n)
{
    for (int i = n - 1; i >= 0; i--) {
        p[i] = (unsigned char)(v & 0xff);
        v >>= 8;
    }
}

static int lime_scan(FILE *f, std::vector<LimeRecord> &recs, bool keep_data)
{
    unsigned char h[144];
    while (true) {
        const size_t n = fread(h, 1, 144, f);
        if (n == 0) break;
        if (n != 144) {
            set_error("LIME: truncated record header");
            return GF_ERR_INVALID;
        }
        const uint32_t magic = ((uint32_t)h[0] << 24) | ((uint32_t)h[1] << 16) | ((uint32_t)h[2] << 8) | h[3];
        if (magic != 0x456789abu) {
            set_error("LIME: bad magic number 0x%08x", magic);
            return GF_ERR_INVALID;
        }
        LimeRecord r;
        r.mb = (h[6] & 0x80) != 0;
        r.me = (h[6] & 0x40) != 0;
        r.length = (long long)be64(h + 8);
        char type[129];
        memcpy(type, h + 16, 128);
        type[128] = 0;
        r.type = type;
        r.offset = ftell(f);
        const long long padded = (r.length + 7) / 8 * 8;
        if (keep_data && r.type != "ildg-binary-data") {
            r.data.resize((size_t)r.length);
            if (r.length && fread(r.data.data(), 1, (size_t)r.length, f) != (size_t)r.length) {
                set_error("LIME: truncated record data");
                return GF_ERR_INVALID;
            }
            if (fseek(f, (long)(padded - r.length), SEEK_CUR)) return GF_ERR_INVALID;
        } else if (fseek(f, (long)padded, SEEK_CUR)) {
            set_error("LIME: truncated record");
            return GF_ERR_INVALID;
        }
        recs.push_back(std::move(r));
    }
    return GF_OK;
}

static bool lime_write_record(FILE *f, const LimeRecord &r, const void *data, long long length)
{
    unsigned char h[144];
    memset(h, 0, sizeof(h));
    put_be(h, 0x456789abu, 4);
    put_be(h + 4, 1, 2);
    h[6] = (unsigned char)((r.mb ? 0x80 : 0) | (r.me ? 0x40 : 0));
    put_be(h + 8, (uint64_t)length, 8);
    strncpy((char *)h + 16, r.type.c_str(), 128);
    if (fwrite(h, 1, 144, f) != 144) return false;
    if (length && fwrite(data, 1, (size_t)length, f) != (size_t)length) return false;
    static const char zeros[8] = {0};
    const long long pad = (length + 7) / 8 * 8 - length;
    return pad == 0 || fwrite(zeros, 1, (size_t)pad, f) == (size_t)pad;
}

struct PinnedBuf {
    void *p = nullptr;
    ~PinnedBuf()
    {
        if (p) cudaFreeHost(p);
    }
};

struct DevBuf {
    void *p = nullptr;
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
};

template <typename Rf>
static int transcode_in(const void *dfile, const Geom &g, const Geom &gs, int order, int swap, int layout, int real,
                        void *dU, cudaStream_t st)
{
    const unsigned blocks = (unsigned)((4 * g.V + 255) / 256);
    if (real == GF_FP64)
        k_file_to_gpu<Rf, double><<<blocks, 256, 0, st>>>((const Rf *)dfile, g, gs, order, swap, layout, (double *)dU);
    else
        k_file_to_gpu<Rf, float><<<blocks, 256, 0, st>>>((const Rf *)dfile, g, gs, order, swap, layout, (float *)dU);
    return launch_status("file transcode");
}

template <typename Rf>
static int transcode_out(const void *dU, const Geom &g, const Geom &gs, int order, int swap, int layout, int real,
                         void *dfile, cudaStream_t st)
{
    const unsigned blocks = (unsigned)((4 * g.V + 255) / 256);
    if (real == GF_FP64)
        k_gpu_to_file<double, Rf><<<blocks, 256, 0, st>>>((const double *)dU, g, gs, order, swap, layout, (Rf *)dfile);
    else
        k_gpu_to_file<float, Rf><<<blocks, 256, 0, st>>>((const float *)dU, g, gs, order, swap, layout, (Rf *)dfile);
    return launch_status("file transcode");
}

// geometry of one timeslice {1, Nx, Ny, Nz} (only used for GF_LAYOUT_TIMESLICE)
static int slice_geom(const int32_t size[4], int layout, Geom &gs)
{
    if (layout != GF_LAYOUT_TIMESLICE) {
        gs = Geom{};
        return GF_OK;
    }
    const int32_t ss[4] = {1, size[1], size[2], size[3]};
    return make_geom(ss, GF_COULOMB, true, gs);
}

}  // namespace gfb

using namespace gfb;

extern "C" {

int gf_file_read(const char *path, int format, int file_real, const int32_t size[4], int real, int layout, void *U,
                 int on_device, void *stream)
{
    clear_error();
    if (!path || !U || !valid_real(real) || !valid_real(file_real) || format < GF_FILE_PLAIN ||
        format > GF_FILE_QCDSTAG || (layout != GF_LAYOUT_GPU && layout != GF_LAYOUT_TIMESLICE)) {
        set_error("invalid argument to gf_file_read");
        return GF_ERR_INVALID;
    }
    Geom g, gs;
    int st = make_geom(size, GF_LANDAU, false, g);
    if (st || (st = slice_geom(size, layout, gs))) return st;
    const bool dbl = (format == GF_FILE_ILDG || format == GF_FILE_QCDSTAG) ? true : file_real == GF_FP64;
    const size_t es = dbl ? 8 : 4;
    const size_t payload = (size_t)g.V * 72 * es;
    FILE *f = fopen(path, "rb");
    if (!f) {
        set_error("cannot open %s", path);
        return GF_ERR_INVALID;
    }
    long long offset = 0;
    if (format == GF_FILE_HEADERONLY) {
        fseek(f, 0, SEEK_END);
        const long long flen = ftell(f);
        offset = flen - (long long)payload;
        if (offset < 0) {
            fclose(f);
            set_error("%s: %lld bytes, smaller than the %zu-byte configuration", path, flen, payload);
            return GF_ERR_INVALID;
        }
    } else if (format == GF_FILE_VOGT) {
        short hd[2];
        if (fread(hd, sizeof(short), 2, f) != 2 || hd[0] != 4 || hd[1] != 3) {
            fclose(f);
            set_error("%s: VOGT header does not describe a 4-dimensional SU(3) field", path);
            return GF_ERR_INVALID;
        }
        short ext[4], lr;
        if (fread(ext, sizeof(short), 4, f) != 4 || fread(&lr, sizeof(short), 1, f) != 1) {
            fclose(f);
            set_error("%s: truncated VOGT header", path);
            return GF_ERR_INVALID;
        }
        for (int i = 0; i < 4; i++)
            if (ext[i] != size[i]) {
                fclose(f);
                set_error("%s: VOGT extents %d %d %d %d do not match the requested lattice", path, ext[0], ext[1],
                          ext[2], ext[3]);
                return GF_ERR_INVALID;
            }
        if ((size_t)lr != es) {
            fclose(f);
            set_error("%s: VOGT header says %d-byte reals, the caller asked for %zu", path, lr, es);
            return GF_ERR_INVALID;
        }
        offset = ftell(f);
    } else if (format == GF_FILE_ILDG) {
        std::vector<LimeRecord> recs;
        if ((st = lime_scan(f, recs, false))) {
            fclose(f);
            return st;
        }
        offset = -1;
        for (auto &r : recs)
            if (r.type == "ildg-binary-data") {
                if ((size_t)r.length != payload) {
                    fclose(f);
                    set_error("%s: ildg-binary-data has %lld bytes, the lattice needs %zu", path, r.length, payload);
                    return GF_ERR_INVALID;
                }
                offset = r.offset;
            }
        if (offset < 0) {
            fclose(f);
            set_error("%s: no ildg-binary-data record", path);
            return GF_ERR_INVALID;
        }
    }
    PinnedBuf host;
    if ((st = cuda_status(cudaHostAlloc(&host.p, payload, cudaHostAllocDefault), "cudaHostAlloc"))) {
        fclose(f);
        return st;
    }
    fseek(f, (long)offset, SEEK_SET);
    const size_t got = fread(host.p, 1, payload, f);
    fclose(f);
    if (got != payload) {
        set_error("%s: truncated (%zu of %zu payload bytes)", path, got, payload);
        return GF_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    DevBuf dfile, dout;
    if ((st = cuda_status(cudaMalloc(&dfile.p, payload), "cudaMalloc"))) return st;
    if ((st = cuda_status(cudaMemcpyAsync(dfile.p, host.p, payload, cudaMemcpyHostToDevice, s), "H2D"))) return st;
    void *dU = U;
    const size_t ubytes = (size_t)g.V * 72 * (real == GF_FP64 ? 8 : 4);
    if (!on_device) {
        if ((st = cuda_status(cudaMalloc(&dout.p, ubytes), "cudaMalloc"))) return st;
        dU = dout.p;
    }
    const int order = format == GF_FILE_ILDG ? ORD_ILDG : (format == GF_FILE_QCDSTAG ? ORD_QCDSTAG : ORD_STANDARD);
    const int swap = format == GF_FILE_ILDG;
    st = dbl ? transcode_in<double>(dfile.p, g, gs, order, swap, layout, real, dU, s)
             : transcode_in<float>(dfile.p, g, gs, order, swap, layout, real, dU, s);
    if (st) return st;
    if (!on_device && (st = cuda_status(cudaMemcpyAsync(U, dU, ubytes, cudaMemcpyDeviceToHost, s), "D2H"))) return st;
    return cuda_status(cudaStreamSynchronize(s), "file read sync");
}

int gf_file_write(const char *path, int format, int file_real, const int32_t size[4], int real, int layout,
                  const void *U, int on_device, const char *template_path, int sa_steps, void *stream)
{
    clear_error();
    if (!path || !U || !valid_real(real) || !valid_real(file_real) || format < GF_FILE_PLAIN ||
        format > GF_FILE_QCDSTAG || (layout != GF_LAYOUT_GPU && layout != GF_LAYOUT_TIMESLICE)) {
        set_error("invalid argument to gf_file_write");
        return GF_ERR_INVALID;
    }
    Geom g, gs;
    int st = make_geom(size, GF_LANDAU, false, g);
    if (st || (st = slice_geom(size, layout, gs))) return st;
    const bool dbl = (format == GF_FILE_ILDG || format == GF_FILE_QCDSTAG) ? true : file_real == GF_FP64;
    const size_t es = dbl ? 8 : 4;
    const size_t payload = (size_t)g.V * 72 * es;
    cudaStream_t s = (cudaStream_t)stream;
    DevBuf din, dfile;
    const void *dU = U;
    const size_t ubytes = (size_t)g.V * 72 * (real == GF_FP64 ? 8 : 4);
    if (!on_device) {
        if ((st = cuda_status(cudaMalloc(&din.p, ubytes), "cudaMalloc"))) return st;
        if ((st = cuda_status(cudaMemcpyAsync(din.p, U, ubytes, cudaMemcpyHostToDevice, s), "H2D"))) return st;
        dU = din.p;
    }
    if ((st = cuda_status(cudaMalloc(&dfile.p, payload), "cudaMalloc"))) return st;
    const int order = format == GF_FILE_ILDG ? ORD_ILDG : (format == GF_FILE_QCDSTAG ? ORD_QCDSTAG : ORD_STANDARD);
    const int swap = format == GF_FILE_ILDG;
    st = dbl ? transcode_out<double>(dU, g, gs, order, swap, layout, real, dfile.p, s)
             : transcode_out<float>(dU, g, gs, order, swap, layout, real, dfile.p, s);
    if (st) return st;
    PinnedBuf host;
    if ((st = cuda_status(cudaHostAlloc(&host.p, payload, cudaHostAllocDefault), "cudaHostAlloc"))) return st;
    if ((st = cuda_status(cudaMemcpyAsync(host.p, dfile.p, payload, cudaMemcpyDeviceToHost, s), "D2H"))) return st;
    if ((st = cuda_status(cudaStreamSynchronize(s), "sync"))) return st;

    // headers / other records from a template file (HEADERONLY, ILDG)
    std::vector<char> header;
    std::vector<LimeRecord> recs;
    if ((format == GF_FILE_HEADERONLY || format == GF_FILE_ILDG) && template_path) {
        FILE *t = fopen(template_path, "rb");
        if (!t) {
            set_error("cannot open template %s", template_path);
            return GF_ERR_INVALID;
        }
        if (format == GF_FILE_HEADERONLY) {
            fseek(t, 0, SEEK_END);
            const long long tl = ftell(t) - (long long)payload;
            if (tl < 0) {
                fclose(t);
                set_error("template %s is smaller than the configuration", template_path);
                return GF_ERR_INVALID;
            }
            header.resize((size_t)tl);
            fseek(t, 0, SEEK_SET);
            if (tl && fread(header.data(), 1, (size_t)tl, t) != (size_t)tl) {
                fclose(t);
                set_error("cannot read the header of %s", template_path);
                return GF_ERR_INVALID;
            }
        } else if ((st = lime_scan(t, recs, true))) {
            fclose(t);
            return st;
        }
        fclose(t);
    }
    FILE *f = fopen(path, "wb");
    if (!f) {
        set_error("cannot create %s", path);
        return GF_ERR_INVALID;
    }
    bool ok = true;
    if (format == GF_FILE_VOGT) {
        const short hd[7] = {4, 3, (short)size[0], (short)size[1], (short)size[2], (short)size[3], (short)es};
        ok = fwrite(hd, sizeof(short), 7, f) == 7;
    } else if (format == GF_FILE_HEADERONLY && !header.empty()) {
        ok = fwrite(header.data(), 1, header.size(), f) == header.size();
    }
    if (format == GF_FILE_ILDG) {
        if (recs.empty()) {  // no template: one self-contained binary record
            LimeRecord r;
            r.type = "ildg-binary-data";
            r.mb = r.me = true;
            recs.push_back(r);
        }
        for (auto &r : recs) {
            if (!ok) break;
            if (r.type == "ildg-binary-data") {
                ok = lime_write_record(f, r, host.p, (long long)payload);
            } else if (r.type == "xlf-info") {
                // the reference appends the number of SA steps (apps/ildg.cpp:196-200)
                std::string txt(r.data.data(), r.data.size());
                txt = std::string(txt.c_str()) + " SA steps " + std::to_string(sa_steps);
                ok = lime_write_record(f, r, txt.data(), (long long)txt.size());
            } else {
                std::string txt(r.data.data(), r.data.size());
                txt = std::string(txt.c_str());  // the reference re-writes text records up to their first NUL
                ok = lime_write_record(f, r, txt.data(), (long long)txt.size());
            }
        }
    } else if (ok) {
        ok = fwrite(host.p, 1, payload, f) == payload;
    }
    if (fclose(f) != 0) ok = false;
    if (!ok) {
        set_error("write error on %s", path);
        return GF_ERR_INVALID;
    }
    return GF_OK;
}

}  // extern "C"
