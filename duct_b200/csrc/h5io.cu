// h5io.cu -- the reference's field checkpoint files uvwp_NNNN.h5:
// save_4fields_fou_hdf5 with h5dump_parallel on one rank and
// writeheader_hdf5 (src/readwrite_hdf5.f90:276-386, 650-722, 851-920), and
// the restart reader read_4fields_fou_hdf5 / h5load_parallel /
// readheader_hdf5 (src/readwrite_hdf5.f90:5-273, 799-849) at the file's own
// y-z resolution.
//
// File content (what the reference's calls create):
//   u, v, w, p   H5T_IEEE_F64BE, HDF5 shape (mx1+1, mz, my, 2): the Fortran
//                array (2, my, mz, mx1+1) of a complex (my, mz, mx1+1) field
//                (src/readwrite_hdf5.f90:311-324, 694);
//   nparams, numerop, mgalx, my, mz, mx1         H5T_STD_I32LE, shape (1);
//   alp, aspect, time, fnu, cfl, dtfixed, cmassflow, SLIP-VELOCITY,
//   DIVERGENCE                                   H5T_IEEE_F64LE, shape (1)
// (h5write_simple_int / h5write_simple_double, :922-968), all in the root
// group.
//
// There is no HDF5 library: the container is written in the HDF5 file
// format directly, in the form libhdf5 gives such a file with its default
// format bounds -- a version 0 superblock, version 1 object headers, the
// root group as a symbol table (a version 1 B-tree of symbol table nodes and
// a local heap of names) and contiguous storage.  The reader takes that
// subset (superblock 0 or 1, symbol-table groups, contiguous or compact
// storage, no filters), which covers files libhdf5 writes that way.
//
// The fields cross in the file's byte order on the GPU: a swap kernel
// writes big-endian doubles straight into mapped pinned host memory, one
// chunk at a time, double-buffered against the file writes; reading runs
// the other way (file -> pinned chunk -> swap kernel -> device field).
#include "internal.h"

#include <errno.h>
#include <fcntl.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <string>
#include <vector>

static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "HDF5 metadata is written as little-endian host words");

namespace duct {

namespace {

constexpr uint64_t kUndef = ~0ull;                 // the undefined address
constexpr uint64_t kHeapFreeNull = 1;              // libhdf5's end of a local heap free list
constexpr int kLeafK = 4, kNodeK = 16;             // group K values of the superblock (libhdf5 defaults)
constexpr size_t kSnodBytes = 8 + 2 * kLeafK * 40;                             // one symbol table node
constexpr size_t kTreeBytes = 24 + 2 * kNodeK * 8 + (2 * kNodeK + 1) * 8;      // one group B-tree node
constexpr size_t kChunkBytes = size_t(8) << 20;    // staged bytes per swap launch
constexpr size_t kFieldAlign = 4096;               // file offset of the first field

inline size_t pad8(size_t x) { return (x + 7) & ~size_t(7); }

// ---------------------------------------------------------------- device

// dst[i] = src[i] with the bytes of each 8-byte word reversed (little- <->
// big-endian doubles); either side may be mapped pinned host memory.
__global__ void k_h5_swap(const unsigned long long *__restrict__ src, unsigned long long *__restrict__ dst,
                          size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const unsigned long long v = src[i];
        const unsigned lo = (unsigned)v, hi = (unsigned)(v >> 32);
        dst[i] = ((unsigned long long)__byte_perm(lo, 0, 0x0123) << 32) | __byte_perm(hi, 0, 0x0123);
    }
}

__global__ void k_h5_copy(const unsigned long long *__restrict__ src, unsigned long long *__restrict__ dst, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

// cheb_interp's sum (src/chebyshev.f90:750-761) for every point (i, j) of
// every mode m: out = sum_{k<K} sum_{l<L} c(k, l, m) ty(i, k) tz(j, l), c the
// old (myr, mzr) planes' Chebyshev coefficients, ty / tz the polynomials at
// the new nodes; the reference's order of summation (k outer, l inner).
__global__ void k_cheb_interp(const double2 *__restrict__ c, double2 *__restrict__ out, const double *__restrict__ ty,
                              const double *__restrict__ tz, int myr, int mzr, int my, int mz, int K, int L, int M)
{
    const long long total = (long long)my * mz * M;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % my);
        const long long r = t / my;
        const int j = (int)(r % mz);
        const long long m = r / mz;
        const double2 *cm = c + (long long)myr * mzr * m;
        double ax = 0.0, ay = 0.0;
        for (int k = 0; k < K; ++k) {
            const double a = ty[(long long)i * K + k];
            for (int l = 0; l < L; ++l) {
                const double2 v = cm[k + (long long)myr * l];
                const double b = tz[(long long)j * L + l];
                ax += v.x * a * b;
                ay += v.y * a * b;
            }
        }
        out[t] = make_double2(ax, ay);
    }
}

int launch_swap(ductgpu_ctx ctx, const void *src, void *dst, size_t words, bool swap)
{
    const size_t blocks = std::min<size_t>((words + 255) / 256, (size_t)ctx->num_sms * 8);
    {
        LaunchScope ls(ctx, DUCTGPU_K_OTHER);
        if (swap)
            k_h5_swap<<<(unsigned)blocks, 256, 0, ctx->stream>>>((const unsigned long long *)src,
                                                                   (unsigned long long *)dst, words);
        else
            k_h5_copy<<<(unsigned)blocks, 256, 0, ctx->stream>>>((const unsigned long long *)src,
                                                                   (unsigned long long *)dst, words);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_h5_swap");
}

// Two mapped pinned chunks and their events, released on every path.
struct Staging {
    void *pin[2] = {};
    void *dev[2] = {};
    cudaEvent_t ev[2] = {};
    ~Staging()
    {
        for (int b = 0; b < 2; ++b) {
            if (ev[b]) {
                cudaEventSynchronize(ev[b]);
                cudaEventDestroy(ev[b]);
            }
        }
        for (int b = 0; b < 2; ++b)
            if (pin[b]) cudaFreeHost(pin[b]);
    }
    int init(ductgpu_ctx ctx)
    {
        for (int b = 0; b < 2; ++b) {
            DUCT_CUDA(ctx, cudaHostAlloc(&pin[b], kChunkBytes, cudaHostAllocMapped));
            DUCT_CUDA(ctx, cudaHostGetDevicePointer(&dev[b], pin[b], 0));
            DUCT_CUDA(ctx, cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming));
        }
        return DUCTGPU_OK;
    }
};

int device_pointer_check(ductgpu_ctx ctx, const void *p, const char *what)
{
    if (!p) return set_error(ctx, DUCTGPU_EARG, "%s: NULL field", what);
    if ((uintptr_t)p & 7) return set_error(ctx, DUCTGPU_EARG, "%s: field not 8-byte aligned", what);
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess || a.type != cudaMemoryTypeDevice) {
        cudaGetLastError();
        return set_error(ctx, DUCTGPU_EARG, "%s: fields must be device memory", what);
    }
    return DUCTGPU_OK;
}

// ---------------------------------------------------------------- writer

enum Kind { kI32, kF64, kF64BE };   // 32-bit int (LE), IEEE double LE, IEEE double BE

// One dataset of a file.  Its data is either given on the host (written
// right after the metadata, 8-byte aligned) or streamed later (`stream`
// >= 0: placed from the next 4 KiB boundary on, in stream order).
struct Dset {
    std::string name;
    Kind kind;
    int rank = 1;
    uint64_t dims[4] = {1, 0, 0, 0};
    const void *host = nullptr;
    int stream = -1;
    uint64_t heap_off = 0, oh = 0, data = 0, bytes = 0;
    uint64_t count() const
    {
        uint64_t n = 1;
        for (int r = 0; r < rank; ++r) n *= dims[r];
        return n;
    }
};

struct Image {
    std::vector<uint8_t> b;
    void u8(size_t o, unsigned v) { b[o] = (uint8_t)v; }
    void u16(size_t o, unsigned v) { memcpy(&b[o], &v, 2); }
    void u32(size_t o, uint32_t v) { memcpy(&b[o], &v, 4); }
    void u64(size_t o, uint64_t v) { memcpy(&b[o], &v, 8); }
    void str(size_t o, const char *s, size_t n) { memcpy(&b[o], s, n); }
    // one version 1 object header message: type, padded body size, flags
    size_t msg(size_t o, unsigned type, unsigned size, unsigned flags)
    {
        u16(o, type);
        u16(o + 2, size);
        u8(o + 4, flags);
        return o + 8;
    }
};

size_t dset_header_bytes(const Dset &d)
{
    return 16 + (8 + 8 + 8 * (size_t)d.rank) + (8 + (d.kind == kI32 ? 16 : 24)) + (8 + 8) + (8 + 24);
}

// The object header of one dataset: dataspace, datatype, fill value (none
// defined, late allocation: libhdf5's defaults), contiguous layout.
void put_dset_header(Image &im, const Dset &d)
{
    const int rank = d.rank;
    const size_t o = d.oh;
    im.u8(o, 1);                                          // object header version 1
    im.u16(o + 2, 4);                                     // messages
    im.u32(o + 4, 1);                                     // reference count
    im.u32(o + 8, (uint32_t)(dset_header_bytes(d) - 16)); // header data bytes
    size_t p = o + 16;
    p = im.msg(p, 0x0001, 8 + 8 * rank, 0);               // dataspace, version 1, no maximum dims
    im.u8(p, 1);
    im.u8(p + 1, rank);
    for (int r = 0; r < rank; ++r) im.u64(p + 8 + 8 * r, d.dims[r]);
    p += 8 + 8 * rank;
    if (d.kind == kI32) {
        p = im.msg(p, 0x0003, 16, 1);                     // datatype: 32-bit signed little-endian
        im.u8(p, 0x10);
        im.u8(p + 1, 0x08);
        im.u32(p + 4, 4);
        im.u16(p + 8, 0);
        im.u16(p + 10, 32);
        p += 16;
    } else {
        p = im.msg(p, 0x0003, 24, 1);                     // datatype: IEEE double
        im.u8(p, 0x11);
        im.u8(p + 1, d.kind == kF64BE ? 0x21 : 0x20);     // implied mantissa msb; byte order
        im.u8(p + 2, 63);                                 // sign bit
        im.u32(p + 4, 8);
        im.u16(p + 8, 0);                                 // bit offset
        im.u16(p + 10, 64);                               // precision
        im.u8(p + 12, 52);                                // exponent location
        im.u8(p + 13, 11);                                // exponent size
        im.u8(p + 14, 0);                                 // mantissa location
        im.u8(p + 15, 52);                                // mantissa size
        im.u32(p + 16, 1023);                             // exponent bias
        p += 24;
    }
    p = im.msg(p, 0x0005, 8, 1);                          // fill value, version 2
    im.u8(p, 2);
    im.u8(p + 1, 2);                                      // allocation time: late
    im.u8(p + 2, 2);                                      // fill write time: if set
    im.u8(p + 3, 0);                                      // no fill value defined
    p += 8;
    p = im.msg(p, 0x0008, 24, 0);                         // data layout, version 3, contiguous
    im.u8(p, 3);
    im.u8(p + 1, 1);
    im.u64(p + 2, d.data);
    im.u64(p + 10, d.bytes);
}

// A whole file but the streamed datasets' data: superblock, root group
// header, local heap, B-tree, symbol table nodes, dataset headers, the host
// datasets' data; the streamed datasets from the next 4 KiB boundary on.
// Sorts ds by name and sets every dataset's address; returns the image and
// the end-of-file address.
void h5_build(std::vector<Dset> &ds, std::vector<uint8_t> &meta, uint64_t &eof)
{
    for (Dset &d : ds) d.bytes = d.count() * (d.kind == kI32 ? 4 : 8);
    // link names in the order the symbol table nodes keep them
    std::sort(ds.begin(), ds.end(), [](const Dset &a, const Dset &b) { return strcmp(a.name.c_str(), b.name.c_str()) < 0; });
    size_t heap_bytes = 8;                                  // offset 0: the empty name
    for (Dset &d : ds) {
        d.heap_off = heap_bytes;
        heap_bytes += pad8(d.name.size() + 1);
    }
    const size_t nsnod = (ds.size() + 2 * kLeafK - 1) / (2 * kLeafK);
    uint64_t a = 96;
    const uint64_t root_oh = a;
    a += 40;
    const uint64_t heap_hdr = a;
    a += 32;
    const uint64_t heap_data = a;
    a += heap_bytes;
    const uint64_t btree = a;
    a += kTreeBytes;
    std::vector<uint64_t> snod(nsnod);
    for (size_t s = 0; s < nsnod; ++s) {
        snod[s] = a;
        a += kSnodBytes;
    }
    for (Dset &d : ds) {
        d.oh = a;
        a += dset_header_bytes(d);
    }
    for (Dset &d : ds)
        if (d.stream < 0) {
            d.data = a;
            a += pad8(d.bytes);
        }
    const uint64_t meta_end = a;
    a = (a + kFieldAlign - 1) / kFieldAlign * kFieldAlign;
    std::vector<Dset *> streamed;
    for (Dset &d : ds)
        if (d.stream >= 0) streamed.push_back(&d);
    std::sort(streamed.begin(), streamed.end(), [](const Dset *x, const Dset *y) { return x->stream < y->stream; });
    for (Dset *d : streamed) {
        d->data = a;
        a += d->bytes;
    }
    eof = streamed.empty() ? meta_end : a;

    Image im;
    im.b.assign(meta_end, 0);
    static const char sig[8] = {'\x89', 'H', 'D', 'F', '\r', '\n', '\x1a', '\n'};
    im.str(0, sig, 8);
    im.u8(13, 8);                                           // size of offsets
    im.u8(14, 8);                                           // size of lengths
    im.u16(16, kLeafK);
    im.u16(18, kNodeK);
    im.u64(24, 0);                                          // base address
    im.u64(32, kUndef);                                     // free-space info
    im.u64(40, eof);
    im.u64(48, kUndef);                                     // driver information
    im.u64(56, 0);                                          // root entry: name offset
    im.u64(64, root_oh);
    im.u32(72, 1);                                          // cache type 1: B-tree and heap cached
    im.u64(80, btree);
    im.u64(88, heap_hdr);
    // root group object header: one symbol table message
    im.u8(root_oh, 1);
    im.u16(root_oh + 2, 1);
    im.u32(root_oh + 4, 1);
    im.u32(root_oh + 8, 24);
    {
        const size_t q = im.msg(root_oh + 16, 0x0011, 16, 0);
        im.u64(q, btree);
        im.u64(q + 8, heap_hdr);
    }
    // local heap of the link names (no free space)
    im.str(heap_hdr, "HEAP", 4);
    im.u64(heap_hdr + 8, heap_bytes);
    im.u64(heap_hdr + 16, kHeapFreeNull);
    im.u64(heap_hdr + 24, heap_data);
    for (const Dset &d : ds) im.str(heap_data + d.heap_off, d.name.c_str(), d.name.size() + 1);
    // one leaf B-tree node over the symbol table nodes; key i+1 is the last
    // name of node i, key 0 the empty name
    im.str(btree, "TREE", 4);
    im.u16(btree + 6, (unsigned)nsnod);
    im.u64(btree + 8, kUndef);
    im.u64(btree + 16, kUndef);
    im.u64(btree + 24, 0);
    for (size_t s = 0; s < nsnod; ++s) {
        const size_t last = std::min(ds.size(), (s + 1) * 2 * kLeafK) - 1;
        im.u64(btree + 32 + 16 * s, snod[s]);
        im.u64(btree + 40 + 16 * s, ds[last].heap_off);
    }
    for (size_t s = 0; s < nsnod; ++s) {
        const size_t lo = s * 2 * kLeafK, hi = std::min(ds.size(), lo + 2 * kLeafK);
        im.str(snod[s], "SNOD", 4);
        im.u8(snod[s] + 4, 1);
        im.u16(snod[s] + 6, (unsigned)(hi - lo));
        for (size_t j = lo; j < hi; ++j) {
            const size_t e = snod[s] + 8 + 40 * (j - lo);
            im.u64(e, ds[j].heap_off);
            im.u64(e + 8, ds[j].oh);
        }
    }
    for (const Dset &d : ds) {
        put_dset_header(im, d);
        if (d.stream < 0 && d.host && d.bytes) memcpy(&im.b[d.data], d.host, d.bytes);
    }
    meta = std::move(im.b);
}

struct FileCloser {
    int fd = -1;
    ~FileCloser()
    {
        if (fd >= 0) close(fd);
    }
};

int pwrite_all(ductgpu_ctx ctx, int fd, const void *buf, size_t n, uint64_t off, const char *path)
{
    const char *p = (const char *)buf;
    while (n) {
        const ssize_t w = pwrite(fd, p, n, (off_t)off);
        if (w < 0 && errno == EINTR) continue;
        if (w <= 0) return set_error(ctx, DUCTGPU_EARG, "write %s: %s", path, strerror(errno));
        p += w;
        n -= (size_t)w;
        off += (uint64_t)w;
    }
    return DUCTGPU_OK;
}

int pread_all(int fd, void *buf, size_t n, uint64_t off)
{
    char *p = (char *)buf;
    while (n) {
        const ssize_t r = pread(fd, p, n, (off_t)off);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) return -1;
        p += r;
        n -= (size_t)r;
        off += (uint64_t)r;
    }
    return 0;
}

// ---------------------------------------------------------------- reader

struct H5Reader {
    ductgpu_ctx ctx = nullptr;
    const char *path = "";
    int fd = -1;
    uint64_t size = 0, base = 0;

    int fail(const char *why)
    {
        return ctx ? set_error(ctx, DUCTGPU_EARG, "%s: %s", path, why) : DUCTGPU_EARG;
    }
    // bytes [addr, addr + n) of the file (relative to the base address)
    bool get(uint64_t addr, void *dst, size_t n)
    {
        if (addr == kUndef || addr > size || n > size || base + addr > size - n) return false;
        return pread_all(fd, dst, n, base + addr) == 0;
    }
    static uint64_t le(const uint8_t *p, int n)
    {
        uint64_t v = 0;
        for (int i = n - 1; i >= 0; --i) v = (v << 8) | p[i];
        return v;
    }

    struct Msg {
        unsigned type;
        std::vector<uint8_t> body;
    };

    // all messages of a version 1 object header, continuation chunks included
    int messages(uint64_t oh, std::vector<Msg> &out)
    {
        uint8_t pre[16];
        if (!get(oh, pre, 16)) return fail("object header outside the file");
        if (!memcmp(pre, "OHDR", 4)) return fail("version 2 object headers are not supported");
        if (pre[0] != 1) return fail("unknown object header version");
        std::vector<std::pair<uint64_t, uint64_t>> chunks{{oh + 16, le(pre + 8, 4)}};
        for (size_t c = 0; c < chunks.size(); ++c) {
            if (chunks.size() > 64) return fail("too many object header continuations");
            const uint64_t len = chunks[c].second;
            if (len > (1u << 20)) return fail("object header chunk too large");
            std::vector<uint8_t> buf(len);
            if (len && !get(chunks[c].first, buf.data(), len)) return fail("object header chunk outside the file");
            size_t p = 0;
            while (p + 8 <= len) {
                const unsigned type = (unsigned)le(&buf[p], 2), sz = (unsigned)le(&buf[p + 2], 2);
                if (p + 8 + sz > len) return fail("object header message overruns its chunk");
                Msg m{type, std::vector<uint8_t>(buf.begin() + p + 8, buf.begin() + p + 8 + sz)};
                if (type == 0x0010) {
                    if (sz < 16) return fail("short continuation message");
                    chunks.push_back({le(m.body.data(), 8), le(m.body.data() + 8, 8)});
                } else if (type != 0) {
                    out.push_back(std::move(m));
                }
                p += 8 + sz;
            }
        }
        return DUCTGPU_OK;
    }

    struct Entry {
        std::string name;
        uint64_t oh;
    };
    std::vector<Entry> entries;
    std::vector<uint8_t> heap;
    int visits = 0;   // B-tree and symbol table nodes read (a bound for cyclic or huge trees)

    int tree(uint64_t addr, int depth)
    {
        if (depth > 16) return fail("group B-tree too deep");
        if (++visits > 65536) return fail("group B-tree too large");
        uint8_t hdr[24];
        if (!get(addr, hdr, 24) || memcmp(hdr, "TREE", 4)) return fail("bad group B-tree node");
        if (hdr[4] != 0) return fail("group B-tree node of another type");
        const int level = hdr[5];
        const unsigned used = (unsigned)le(hdr + 6, 2);
        if (used > 4096) return fail("group B-tree node too large");
        std::vector<uint8_t> kc(used * 16 + 8);
        if (!get(addr + 24, kc.data(), kc.size())) return fail("group B-tree node outside the file");
        for (unsigned i = 0; i < used; ++i) {
            const uint64_t child = le(&kc[8 + 16 * i], 8);
            if (level > 0) {
                if (int rc = tree(child, depth + 1)) return rc;
                continue;
            }
            uint8_t sh[8];
            if (++visits > 65536) return fail("group B-tree too large");
            if (!get(child, sh, 8) || memcmp(sh, "SNOD", 4)) return fail("bad symbol table node");
            const unsigned n = (unsigned)le(sh + 6, 2);
            if (n > 4096) return fail("symbol table node too large");
            std::vector<uint8_t> e(40 * (size_t)n);
            if (n && !get(child + 8, e.data(), e.size())) return fail("symbol table node outside the file");
            for (unsigned j = 0; j < n; ++j) {
                const uint64_t off = le(&e[40 * j], 8);
                if (off >= heap.size()) return fail("link name outside the local heap");
                const uint8_t *s = heap.data() + off;
                const size_t len = strnlen((const char *)s, heap.size() - off);
                if (off + len >= heap.size()) return fail("unterminated link name");
                entries.push_back({std::string((const char *)s, len), le(&e[40 * j + 8], 8)});
            }
        }
        return DUCTGPU_OK;
    }

    int open_root()
    {
        struct stat st;
        if (fstat(fd, &st) != 0) return fail("cannot stat");
        size = (uint64_t)st.st_size;
        // the superblock sits at 0 or after a user block of 512 * 2^k bytes
        static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
        uint64_t at = kUndef;
        for (uint64_t o = 0; o + 8 <= size; o = o ? 2 * o : 512) {
            uint8_t s[8];
            if (pread_all(fd, s, 8, o) == 0 && !memcmp(s, sig, 8)) {
                at = o;
                break;
            }
        }
        if (at == kUndef) return fail("not an HDF5 file");
        uint8_t sb[104];
        if (at + 96 > size || pread_all(fd, sb, std::min<uint64_t>(sizeof sb, size - at), at) != 0)
            return fail("truncated superblock");
        const int ver = sb[8];
        if (ver > 1) return fail("superblock versions 2 and 3 are not supported");
        if (sb[13] != 8 || sb[14] != 8) return fail("only 8-byte offsets and lengths are supported");
        const size_t q = ver == 1 ? 28 : 24;            // version 1 adds the indexed storage K
        if (at + q + 72 > size) return fail("truncated superblock");
        base = le(sb + q, 8);
        if (base != at && base != 0) return fail("unexpected base address");
        base = at;
        const uint64_t eof = le(sb + q + 16, 8);
        if (eof != kUndef && base + eof > size) return fail("truncated file (shorter than its end-of-file address)");
        const uint8_t *root = sb + q + 32;               // root group symbol table entry
        std::vector<Msg> ms;
        if (int rc = messages(le(root + 8, 8), ms)) return rc;
        uint64_t bt = kUndef, hp = kUndef;
        for (const Msg &m : ms)
            if (m.type == 0x0011 && m.body.size() >= 16) {
                bt = le(m.body.data(), 8);
                hp = le(m.body.data() + 8, 8);
            }
        if (bt == kUndef) return fail("the root group is not a symbol-table group");
        uint8_t hh[32];
        if (!get(hp, hh, 32) || memcmp(hh, "HEAP", 4)) return fail("bad local heap");
        const uint64_t hsz = le(hh + 8, 8), haddr = le(hh + 24, 8);
        if (hsz > (64u << 20)) return fail("local heap too large");
        heap.resize(hsz);
        if (hsz && !get(haddr, heap.data(), hsz)) return fail("local heap outside the file");
        return tree(bt, 0);
    }

    // a dataset's shape, element type and storage
    struct Info {
        int rank = -1;
        uint64_t dims[8] = {};
        int cls = -1, tsize = 0, big = 0, sgn = 1;
        int layout = -1;                    // 0 compact, 1 contiguous
        uint64_t addr = kUndef, bytes = 0;
        std::vector<uint8_t> compact;
        uint64_t count() const
        {
            uint64_t n = 1;
            for (int r = 0; r < rank; ++r) n *= dims[r];
            return n;
        }
    };

    // DUCTGPU_OK, an error status, or kMissing for an absent optional dataset
    static constexpr int kMissing = -1;
    int info(const std::string &name, Info &I, bool required = true)
    {
        const Entry *e = nullptr;
        for (const Entry &x : entries)
            if (x.name == name) e = &x;
        if (!e) {
            if (!required) return kMissing;
            std::string w = "no dataset '" + name + "'";
            return fail(w.c_str());
        }
        std::vector<Msg> ms;
        if (int rc = messages(e->oh, ms)) return rc;
        for (const Msg &m : ms) {
            const uint8_t *b = m.body.data();
            const size_t n = m.body.size();
            if (m.type == 0x0001 && n >= 4) {
                const int v = b[0];
                I.rank = b[1];
                if (I.rank > 8) return fail("dataspace rank above 8");
                const size_t at = v == 1 ? 8 : 4;
                if (v == 2 && b[3] == 2) return fail("null dataspace");
                if (n < at + 8 * (size_t)I.rank) return fail("short dataspace message");
                for (int r = 0; r < I.rank; ++r) I.dims[r] = le(b + at + 8 * r, 8);
            } else if (m.type == 0x0003 && n >= 8) {
                I.cls = b[0] & 0x0f;
                I.big = b[1] & 1;
                I.sgn = (b[1] >> 3) & 1;
                I.tsize = (int)le(b + 4, 4);
                if (I.cls == 1 && (b[1] & 0x40)) return fail("VAX floating point is not supported");
            } else if (m.type == 0x0008 && n >= 2) {
                const int v = b[0];
                if (v == 3 || v == 4) {
                    I.layout = b[1];
                    if (I.layout == 0 && n >= 4) {
                        const size_t cs = (size_t)le(b + 2, 2);
                        if (n < 4 + cs) return fail("short compact layout");
                        I.compact.assign(b + 4, b + 4 + cs);
                    } else if (I.layout == 1 && n >= 18) {
                        I.addr = le(b + 2, 8);
                        I.bytes = le(b + 10, 8);
                    } else {
                        return fail("chunked or virtual storage is not supported");
                    }
                } else if ((v == 1 || v == 2) && n >= 16 && b[2] == 1) {
                    I.layout = 1;
                    I.addr = le(b + 8, 8);
                    I.bytes = kUndef;
                } else {
                    return fail("unsupported data layout message");
                }
            } else if (m.type == 0x000b) {
                return fail("filtered (compressed) datasets are not supported");
            }
        }
        if (I.rank < 0 || I.cls < 0 || I.layout < 0) return fail("dataset without dataspace, datatype or layout");
        if (I.layout == 1 && I.bytes == kUndef) I.bytes = I.count() * (uint64_t)I.tsize;
        return DUCTGPU_OK;
    }

    // the first element of a scalar dataset as a double / an int
    int scalar(const std::string &name, double *d, long long *i, bool required = true)
    {
        Info I;
        if (int rc = info(name, I, required)) return rc;
        if (I.count() < 1 || I.tsize < 1 || I.tsize > 8) return fail("bad scalar dataset");
        uint8_t raw[8];
        if (I.layout == 0) {
            if (I.compact.size() < (size_t)I.tsize) return fail("short compact scalar");
            memcpy(raw, I.compact.data(), I.tsize);
        } else if (I.addr == kUndef || !get(I.addr, raw, I.tsize)) {
            return fail("scalar data outside the file");
        }
        if (I.big) std::reverse(raw, raw + I.tsize);
        if (I.cls == 1) {
            double v;
            if (I.tsize == 8) memcpy(&v, raw, 8);
            else if (I.tsize == 4) { float f; memcpy(&f, raw, 4); v = f; }
            else return fail("unsupported float size");
            if (d) *d = v;
            if (i) *i = (long long)v;
        } else if (I.cls == 0) {
            uint64_t u = le(raw, I.tsize);
            long long v = (long long)u;
            if (I.sgn && I.tsize < 8 && (u >> (8 * I.tsize - 1)) & 1) v = (long long)(u | (~0ull << (8 * I.tsize)));
            if (d) *d = (double)v;
            if (i) *i = v;
        } else {
            return fail("scalar of an unsupported class");
        }
        return DUCTGPU_OK;
    }
};

struct ReaderFile {
    H5Reader r;
    ~ReaderFile()
    {
        if (r.fd >= 0) close(r.fd);
    }
};

int read_header(H5Reader &r, ductgpu_h5_header *h)
{
    memset(h, 0, sizeof *h);
    long long v;
    double x;
    if (int rc = r.scalar("nparams", nullptr, &v)) return rc;
    h->nparams = (int)v;
    int rc = r.scalar("numerop", nullptr, &v, false);
    if (rc > 0) return rc;
    h->numerop = rc == 0 ? (int)v : 1;
    if (int rc = r.scalar("mgalx", nullptr, &v)) return rc;
    h->mgalx = (int)v;
    if (int rc = r.scalar("my", nullptr, &v)) return rc;
    h->my = (int)v;
    if (int rc = r.scalar("mz", nullptr, &v)) return rc;
    h->mz = (int)v;
    // readheader_hdf5 (src/readwrite_hdf5.f90:822-825): without mx1 the
    // file is taken to hold the 2/3-rule modes of mgalx
    rc = r.scalar("mx1", nullptr, &v, false);
    if (rc > 0) return rc;
    h->mx1 = rc == 0 ? (int)v : 2 * (h->mgalx / 3) / 2 - 1;
    struct {
        const char *name;
        double *dst;
    } dbl[] = {{"alp", &h->alp}, {"aspect", &h->aspect}, {"time", &h->time}, {"fnu", &h->fnu},
               {"cfl", &h->cfl}, {"dtfixed", &h->dtfixed}, {"cmassflow", &h->cmassflow},
               {"SLIP-VELOCITY", &h->slip}, {"DIVERGENCE", &h->divergence}};
    for (auto &e : dbl) {
        const int rq = r.scalar(e.name, &x, nullptr, false);
        if (rq > 0) return rq;
        if (rq == 0) *e.dst = x;
    }
    return DUCTGPU_OK;
}

} // namespace

// The metadata of a uvwp_NNNN.h5 file -- everything before the four fields'
// data -- and where the fields go.  Layout: superblock, root group header,
// local heap, B-tree, symbol table nodes, dataset headers, the scalars'
// data, then u, v, w, p from the next 4 KiB boundary on.
// A file whose datasets all come from the host.
int h5_write_host(ductgpu_ctx ctx, const char *filename, std::vector<Dset> &ds)
{
    std::vector<uint8_t> img;
    uint64_t eof = 0;
    h5_build(ds, img, eof);
    FileCloser fc;
    fc.fd = open(filename, O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (fc.fd < 0) return set_error(ctx, DUCTGPU_EARG, "open %s: %s", filename, strerror(errno));
    if (int rc = pwrite_all(ctx, fc.fd, img.data(), img.size(), 0, filename)) return rc;
    const int fd = fc.fd;
    fc.fd = -1;
    if (close(fd) != 0) return set_error(ctx, DUCTGPU_EARG, "close %s: %s", filename, strerror(errno));
    return DUCTGPU_OK;
}

// write_statistics_hdf5 (src/readwrite_hdf5.f90:388-648, one rank, no
// temperature): the statistics accumulated over nstat recorded steps as the
// reference names and shapes them.  Host arrays in the stepper's layout:
// mean [4][P] (u, v, w, p), prod [6][P] (uu, vv, ww, uv, uw, vw), ppb [P],
// spec [4][7][M], om2 [3][P]; P = my mz.
int h5_write_statistics(ductgpu_ctx ctx, const char *filename, const H5Stats &st)
{
    const uint64_t P = (uint64_t)st.my * st.mz;
    const int32_t iv[4] = {st.mgalx, st.my, st.mz, st.nstat};
    const char *in[4] = {"mgalx", "my", "mz", "nstat"};
    const double dv[5] = {st.timef, st.time, st.fnu, st.alp, st.aspect};
    const char *dn[5] = {"timef", "time", "fnu", "alp", "aspect"};
    // the seven spectra points of statistics_fou (src/operators.F:1680-1693), 1-based
    const int32_t jinco[7] = {st.my / 16, st.my / 8, st.my / 4, st.my / 2, st.my / 16, st.my / 8, st.my / 4};
    const int32_t kinco[7] = {st.mz / 2, st.mz / 2, st.mz / 2, st.mz / 2, st.mz / 16, st.mz / 8, st.mz / 4};
    std::vector<Dset> ds;
    auto scalar = [&](const char *n, Kind k, const void *v) {
        Dset d{n, k};
        d.host = v;
        ds.push_back(d);
    };
    auto plane = [&](const char *n, const double *v) {    // Fortran (my, mz): HDF5 (mz, my)
        Dset d{n, kF64};
        d.rank = 2;
        d.dims[0] = (uint64_t)st.mz;
        d.dims[1] = (uint64_t)st.my;
        d.host = v;
        ds.push_back(d);
    };
    for (int i = 0; i < 4; ++i) scalar(in[i], kI32, &iv[i]);
    for (int i = 0; i < 5; ++i) scalar(dn[i], kF64, &dv[i]);
    const char *mn[4] = {"um", "vm", "wm", "pm"};
    for (int c = 0; c < 4; ++c) plane(mn[c], st.mean + c * P);
    const char *pn[6] = {"uub", "vvb", "wwb", "uvb", "uwb", "vwb"};
    for (int c = 0; c < 6; ++c) plane(pn[c], st.prod + c * P);
    plane("ppb", st.ppb);
    const char *on[3] = {"ox2", "oy2", "oz2"};
    for (int c = 0; c < 3; ++c) plane(on[c], st.om2 + c * P);
    const char *sn[4] = {"uust", "vvst", "wwst", "ppst"};
    for (int c = 0; c < 4; ++c) {                       // Fortran (0:mx1, nspec): HDF5 (nspec, mx1+1)
        Dset d{sn[c], kF64};
        d.rank = 2;
        d.dims[0] = 7;
        d.dims[1] = (uint64_t)st.nmodes;
        d.host = st.spec + (size_t)c * 7 * st.nmodes;
        ds.push_back(d);
    }
    for (int t = 0; t < 2; ++t) {
        Dset d{t ? "kinco" : "jinco", kI32};
        d.dims[0] = 7;
        d.host = t ? kinco : jinco;
        ds.push_back(d);
    }
    return h5_write_host(ctx, filename, ds);
}

void h5_layout(const ductgpu_h5_header *hdr, H5Layout &L)
{
    const uint64_t nm = (uint64_t)hdr->mx1 + 1;
    // writeheader_hdf5's scalars (nparams 7: no temperature) and the fields
    const int32_t iv[6] = {7, hdr->numerop > 0 ? hdr->numerop : 1, hdr->mgalx, hdr->my, hdr->mz, hdr->mx1};
    const char *in[6] = {"nparams", "numerop", "mgalx", "my", "mz", "mx1"};
    const double dv[9] = {hdr->alp, hdr->aspect, hdr->time, hdr->fnu, hdr->cfl, hdr->dtfixed, hdr->cmassflow,
                          hdr->slip, hdr->divergence};
    const char *dn[9] = {"alp", "aspect", "time", "fnu", "cfl", "dtfixed", "cmassflow", "SLIP-VELOCITY", "DIVERGENCE"};
    std::vector<Dset> ds;
    for (int i = 0; i < 6; ++i) {
        Dset d{in[i], kI32};
        d.host = &iv[i];
        ds.push_back(d);
    }
    for (int i = 0; i < 9; ++i) {
        Dset d{dn[i], kF64};
        d.host = &dv[i];
        ds.push_back(d);
    }
    const char *fname[4] = {"u", "v", "w", "p"};
    for (int f = 0; f < 4; ++f) {
        Dset d{fname[f], kF64BE};
        d.rank = 4;
        d.dims[0] = nm;
        d.dims[1] = (uint64_t)hdr->mz;
        d.dims[2] = (uint64_t)hdr->my;
        d.dims[3] = 2;
        d.stream = f;
        ds.push_back(d);
    }
    h5_build(ds, L.meta, L.eof);
    for (const Dset &d : ds)
        if (d.stream >= 0) {
            L.field_off[d.stream] = d.data;
            L.field_bytes = d.bytes;
        }
}

} // namespace duct

using namespace duct;

extern "C" int ductgpu_uvwp_filename(const char *fuvwpout, int iimag, char *out, int cap)
{
    if (!fuvwpout || !out || cap <= 0) return DUCTGPU_EARG;
    // concat5b (src/concat.F:74-87): the prefix up to its first blank, then
    // 'uvwp_', iimag as Fortran i4.4 (asterisks when it does not fit), '.h5'
    std::string s(fuvwpout);
    const size_t sp = s.find(' ');
    if (sp != std::string::npos) s.resize(sp);
    char num[16];
    if (iimag >= 0 && iimag <= 9999) snprintf(num, sizeof num, "%04d", iimag);
    else snprintf(num, sizeof num, "****");
    s += "uvwp_";
    s += num;
    s += ".h5";
    if ((int)s.size() + 1 > cap) return DUCTGPU_EARG;
    memcpy(out, s.c_str(), s.size() + 1);
    return DUCTGPU_OK;
}

extern "C" int ductgpu_statistics_filename(const char *fuvwpout, char *out, int cap)
{
    if (!fuvwpout || !out || cap <= 0) return DUCTGPU_EARG;
    // concatb(fuvwpout,'statistics_',11,ext,4,'.h5',3,filename) with ext the
    // i4.4 of the first icf = 1, 2, ... whose file does not exist
    // (src/readwrite_hdf5.f90:446-456, src/concat.F:33-45)
    std::string head(fuvwpout);
    const size_t sp = head.find(' ');
    if (sp != std::string::npos) head.resize(sp);
    for (int icf = 1; icf <= 9999; ++icf) {
        char num[16];
        snprintf(num, sizeof num, "%04d", icf);
        const std::string s = head + "statistics_" + num + ".h5";
        if (access(s.c_str(), F_OK) == 0) continue;
        if ((int)s.size() + 1 > cap) return DUCTGPU_EARG;
        memcpy(out, s.c_str(), s.size() + 1);
        return DUCTGPU_OK;
    }
    return DUCTGPU_EARG;   // all 9999 taken (the reference would loop for ever)
}

extern "C" int ductgpu_save_4fields_fou_hdf5_dev(ductgpu_ctx ctx, const char *filename, const double *u,
                                                 const double *v, const double *w, const double *p,
                                                 const ductgpu_h5_header *hdr)
{
    if (!ctx) return DUCTGPU_EARG;
    if (!filename || !hdr) return set_error(ctx, DUCTGPU_EARG, "save_4fields_fou_hdf5: NULL argument");
    if (ctx->capturing) return set_error(ctx, DUCTGPU_ESTATE, "save_4fields_fou_hdf5: inside a graph capture");
    cudaSetDevice(ctx->device);
    if (hdr->my < 1 || hdr->mz < 1 || hdr->mx1 < 0 || hdr->my > 65536 || hdr->mz > 65536 || hdr->mx1 > 65535)
        return set_error(ctx, DUCTGPU_EARG, "save_4fields_fou_hdf5: bad sizes my %d mz %d mx1 %d", hdr->my,
                         hdr->mz, hdr->mx1);
    const double *fields[4] = {u, v, w, p};
    for (int f = 0; f < 4; ++f)
        if (int rc = device_pointer_check(ctx, fields[f], "save_4fields_fou_hdf5")) return rc;
    H5Layout L;
    h5_layout(hdr, L);
    const uint64_t fbytes = L.field_bytes;

    FileCloser fc;
    fc.fd = open(filename, O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (fc.fd < 0) return set_error(ctx, DUCTGPU_EARG, "open %s: %s", filename, strerror(errno));
    if (int rc = pwrite_all(ctx, fc.fd, L.meta.data(), L.meta.size(), 0, filename)) return rc;

    // the fields: big-endian on the GPU into pinned chunk b, written while
    // the next chunk is converted
    Staging st;
    if (int rc = st.init(ctx)) return rc;
    struct Piece {
        const char *src;
        uint64_t off, bytes;
    };
    std::vector<Piece> pieces;
    for (int f = 0; f < 4; ++f)
        for (uint64_t o = 0; o < fbytes; o += kChunkBytes)
            pieces.push_back({(const char *)fields[f] + o, L.field_off[f] + o, std::min<uint64_t>(kChunkBytes, fbytes - o)});
    for (size_t k = 0; k <= pieces.size(); ++k) {
        if (k < pieces.size()) {
            const int b = (int)(k & 1);
            if (int rc = launch_swap(ctx, pieces[k].src, st.dev[b], pieces[k].bytes / 8, true)) return rc;
            DUCT_CUDA(ctx, cudaEventRecord(st.ev[b], ctx->stream));
        }
        if (k > 0) {
            const int b = (int)((k - 1) & 1);
            DUCT_CUDA(ctx, cudaEventSynchronize(st.ev[b]));
            if (int rc = pwrite_all(ctx, fc.fd, st.pin[b], pieces[k - 1].bytes, pieces[k - 1].off, filename)) return rc;
        }
    }
    if (close(fc.fd) != 0) {
        fc.fd = -1;
        return set_error(ctx, DUCTGPU_EARG, "close %s: %s", filename, strerror(errno));
    }
    fc.fd = -1;
    return DUCTGPU_OK;
}

extern "C" int ductgpu_read_hdf5_header(ductgpu_ctx ctx, const char *filename, ductgpu_h5_header *hdr)
{
    if (!filename || !hdr) return ctx ? set_error(ctx, DUCTGPU_EARG, "read_hdf5_header: NULL argument") : DUCTGPU_EARG;
    ReaderFile rf;
    rf.r.ctx = ctx;
    rf.r.path = filename;
    rf.r.fd = open(filename, O_RDONLY);
    if (rf.r.fd < 0) return ctx ? set_error(ctx, DUCTGPU_EARG, "open %s: %s", filename, strerror(errno)) : DUCTGPU_EARG;
    if (int rc = rf.r.open_root()) return rc;
    return read_header(rf.r, hdr);
}

extern "C" int ductgpu_read_4fields_fou_hdf5_dev(ductgpu_ctx ctx, const char *filename, double *u, double *v,
                                                 double *w, double *p, int my, int mz, int nmodes,
                                                 ductgpu_h5_header *hdr_out)
{
    if (!ctx) return DUCTGPU_EARG;
    if (!filename) return set_error(ctx, DUCTGPU_EARG, "read_4fields_fou_hdf5: NULL file name");
    if (ctx->capturing) return set_error(ctx, DUCTGPU_ESTATE, "read_4fields_fou_hdf5: inside a graph capture");
    cudaSetDevice(ctx->device);
    if (my < 1 || mz < 1 || nmodes < 1) return set_error(ctx, DUCTGPU_EARG, "read_4fields_fou_hdf5: bad sizes");
    double *fields[4] = {u, v, w, p};
    for (int f = 0; f < 4; ++f)
        if (int rc = device_pointer_check(ctx, fields[f], "read_4fields_fou_hdf5")) return rc;
    ReaderFile rf;
    H5Reader &r = rf.r;
    r.ctx = ctx;
    r.path = filename;
    r.fd = open(filename, O_RDONLY);
    if (r.fd < 0) return set_error(ctx, DUCTGPU_EARG, "open %s: %s", filename, strerror(errno));
    if (int rc = r.open_root()) return rc;
    ductgpu_h5_header h;
    if (int rc = read_header(r, &h)) return rc;
    // read_4fields_fou_hdf5 (src/readwrite_hdf5.f90:129-136): another my AND
    // mz re-interpolates every plane (cheb_interp); the reference's copy for
    // one of them alone reads outside its array, so that is refused here
    const bool interp = h.my != my || h.mz != mz;
    if (interp && (h.my == my || h.mz == mz))
        return set_error(ctx, DUCTGPU_EARG,
                         "%s holds my %d mz %d, asked for my %d mz %d: only both sizes changed re-interpolate",
                         filename, h.my, h.mz, my, mz);
    if (interp && (h.my < 2 || h.mz < 2 || h.my > 4097 || h.mz > 4097))
        return set_error(ctx, DUCTGPU_EARG, "%s: my %d mz %d", filename, h.my, h.mz);
    // the old planes' Chebyshev transform needs n - 1 = 2^a 3^b (checked
    // here, before anything is written to the fields)
    auto dct_len_ok = [](int n) {
        int m = n - 1;
        while (m % 2 == 0) m /= 2;
        while (m % 3 == 0) m /= 3;
        return m == 1;
    };
    if (interp && (!dct_len_ok(h.my) || !dct_len_ok(h.mz)))
        return set_error(ctx, DUCTGPU_EARG, "%s: my %d mz %d cannot be re-interpolated (n - 1 must be 2^a 3^b)",
                         filename, h.my, h.mz);
    const int fy = interp ? h.my : my, fz = interp ? h.mz : mz;   // the file's planes
    const char *fname[4] = {"u", "v", "w", "p"};
    const uint64_t fplane = (uint64_t)fy * fz * 16;
    struct Piece {
        int f;
        uint64_t dst, off, bytes;
        bool swap;
    };
    std::vector<Piece> pieces;
    uint64_t kept[4] = {};
    for (int f = 0; f < 4; ++f) {
        H5Reader::Info I;
        if (int rc = r.info(fname[f], I)) return rc;
        if (I.cls != 1 || I.tsize != 8) return set_error(ctx, DUCTGPU_EARG, "%s: %s is not double", filename, fname[f]);
        if (I.rank != 4 || I.dims[1] != (uint64_t)fz || I.dims[2] != (uint64_t)fy || I.dims[3] != 2)
            return set_error(ctx, DUCTGPU_EARG, "%s: %s is not (modes, %d, %d, 2)", filename, fname[f], fz, fy);
        if (I.layout != 1 || I.addr == kUndef || I.bytes != I.count() * 8)
            return set_error(ctx, DUCTGPU_EARG, "%s: %s is not contiguous", filename, fname[f]);
        // h5load_parallel + the copy of read_4fields_fou_hdf5: the file's
        // modes beyond nmodes are dropped, missing ones are zero
        const uint64_t keep = std::min<uint64_t>(I.dims[0], (uint64_t)nmodes) * fplane;
        if (r.base + I.addr > r.size || keep > r.size - (r.base + I.addr))
            return set_error(ctx, DUCTGPU_EARG, "%s: %s data outside the file", filename, fname[f]);
        for (uint64_t o = 0; o < keep; o += kChunkBytes)
            pieces.push_back({f, o, r.base + I.addr + o, std::min<uint64_t>(kChunkBytes, keep - o), I.big != 0});
        kept[f] = keep;
    }
    const uint64_t kmodes = kept[0] / fplane;
    for (int f = 1; f < 4; ++f)
        if (kept[f] != kept[0]) return set_error(ctx, DUCTGPU_EARG, "%s: u, v, w, p differ in modes", filename);
    // the file's planes go straight to the fields, or to a scratch array
    // of the file's size when they are re-interpolated
    struct Scratch {
        void *p[3] = {};
        ~Scratch()
        {
            for (void *q : p)
                if (q) cudaFree(q);
        }
    } sc;
    double *raw = nullptr;
    const uint64_t fbytes = kmodes * fplane;
    if (interp && fbytes) {
        if (cudaMalloc(&sc.p[0], 4 * fbytes) != cudaSuccess) {
            cudaGetLastError();
            return set_error(ctx, DUCTGPU_EALLOC, "read_4fields_fou_hdf5: %.1f MB of re-interpolation scratch",
                             4.0 * fbytes / 1e6);
        }
        raw = (double *)sc.p[0];
    }
    // nothing is written to the fields before all four checked out
    const uint64_t plane = (uint64_t)my * mz * 16;
    const uint64_t done = interp ? 0 : kept[0];
    for (int f = 0; f < 4; ++f)
        if (done < (uint64_t)nmodes * plane)
            DUCT_CUDA(ctx, cudaMemsetAsync((char *)fields[f] + done, 0, (uint64_t)nmodes * plane - done, ctx->stream));
    Staging st;
    if (int rc = st.init(ctx)) return rc;
    for (size_t k = 0; k < pieces.size(); ++k) {
        const int b = (int)(k & 1);
        if (k >= 2) DUCT_CUDA(ctx, cudaEventSynchronize(st.ev[b]));   // the launch that read chunk b is done
        if (pread_all(r.fd, st.pin[b], pieces[k].bytes, pieces[k].off) != 0)
            return set_error(ctx, DUCTGPU_EARG, "read %s: %s", filename, strerror(errno));
        char *base = interp ? (char *)raw + pieces[k].f * fbytes : (char *)fields[pieces[k].f];
        if (int rc = launch_swap(ctx, st.dev[b], base + pieces[k].dst, pieces[k].bytes / 8, pieces[k].swap)) return rc;
        DUCT_CUDA(ctx, cudaEventRecord(st.ev[b], ctx->stream));
    }
    if (interp && kmodes) {
        // cheb_interp (src/chebyshev.f90:725-765) of every plane: its
        // Chebyshev coefficients (transyz_plane_fou -1), the first
        // min(20, myr) x min(20, mzr) of them summed at the new nodes
        for (int f = 0; f < 4; ++f) {
            double *q = (double *)((char *)raw + f * fbytes);
            if (int rc = transyz_dev(ctx, q, fy, fz, (int)kmodes, 'y', -1)) return rc;
            if (int rc = transyz_dev(ctx, q, fy, fz, (int)kmodes, 'z', -1)) return rc;
        }
        const int K = std::min(20, fy), L = std::min(20, fz);
        std::vector<double> t((size_t)my * K + (size_t)mz * L);
        // cos(k acos(y2)) with y2 = -dglc(-1, 1, my) (src/chebyshev.f90:429-456)
        const double pi = 4.0 * atan(1.0);
        for (int i = 0; i < my; ++i) {
            const double y2 = -(-cos((double)i * (pi / (double)(my - 1))));
            for (int k = 0; k < K; ++k) t[(size_t)i * K + k] = cos((double)k * acos(y2));
        }
        for (int j = 0; j < mz; ++j) {
            const double z2 = -(-cos((double)j * (pi / (double)(mz - 1))));
            for (int l = 0; l < L; ++l) t[(size_t)my * K + (size_t)j * L + l] = cos((double)l * acos(z2));
        }
        if (cudaMalloc(&sc.p[1], t.size() * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            return set_error(ctx, DUCTGPU_EALLOC, "read_4fields_fou_hdf5: interpolation tables");
        }
        const double *ty = (const double *)sc.p[1];
        DUCT_CUDA(ctx, cudaMemcpyAsync(sc.p[1], t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice,
                                       ctx->stream));
        for (int f = 0; f < 4; ++f) {
            const long long total = (long long)my * mz * (long long)kmodes;
            const int blocks = (int)std::min<long long>((total + 255) / 256, (long long)ctx->num_sms * 16);
            {
                LaunchScope ls(ctx, DUCTGPU_K_OTHER);
                k_cheb_interp<<<blocks, 256, 0, ctx->stream>>>(
                    reinterpret_cast<const double2 *>((char *)raw + f * fbytes), reinterpret_cast<double2 *>(fields[f]),
                    ty, ty + (size_t)my * K, fy, fz, my, mz, K, L, (int)kmodes);
            }
            DUCT_CUDA(ctx, cudaGetLastError());
        }
        // the scratch is freed (and the tables) only after the kernels
        DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    if (hdr_out) *hdr_out = h;
    return DUCTGPU_OK;
}
