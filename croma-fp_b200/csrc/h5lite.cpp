// h5lite.cpp -- reader of the HDF5 tracer snapshots CROMA takes as input
// (the reference's tracer_10k/subset__tracer_z_dumpNNNN.h5; read there by
// libhdf5 in tracer_load_hdf5_raw_snapshot_slice,
// src/tracer_fp_background.c:1003-1204, and read_redshift_hdf5, :70-146).
//
// libhdf5 is not linked into this library, so this file reads the subset of the
// HDF5 format (File Format Specification version 3.0) that those files use:
//   * superblock version 0 or 1 (signature at offset 0 or at a user-block
//     boundary 512 * 2^k), 8-byte offsets and lengths;
//   * groups stored as symbol tables: version-1 B-tree group nodes ("TREE"),
//     symbol table nodes ("SNOD") and a local heap ("HEAP") for the names;
//     nested groups are followed through '/'-separated paths;
//   * version-1 object headers, with continuation blocks;
//   * datasets with a version 1 or 2 dataspace, a fixed-point (1/2/4/8-byte,
//     signed or unsigned) or IEEE floating-point (4/8-byte) datatype in either
//     byte order, and a version 3 or 4 layout message of class compact or
//     contiguous; no filter pipeline.
// Anything else -- superblock 2/3, version-2 object headers, link messages,
// chunked or filtered storage, other datatype classes -- is refused with an
// error that names it.  Every offset read from the file is checked against
// the file's size before it is used.
#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include "../../include/croma_b200.h"

namespace croma {
void set_error(const std::string &msg);   // api.cu
}
using croma::set_error;

namespace {

constexpr uint64_t kUndef = ~0ull;

struct H5Error {
    std::string msg;
};

[[noreturn]] void fail(const std::string &m) { throw H5Error{m}; }

struct File {
    int fd = -1;
    uint64_t size = 0;
    uint64_t base = 0;   // base address: file addresses are relative to it
    int so = 8, sl = 8;  // sizes of offsets and lengths
    std::string path;

    explicit File(const char *p) : path(p)
    {
        fd = ::open(p, O_RDONLY);
        if (fd < 0) fail("cannot open '" + path + "': " + std::strerror(errno));
        struct stat st;
        if (fstat(fd, &st) != 0) fail("cannot stat '" + path + "'");
        size = (uint64_t)st.st_size;
    }
    ~File()
    {
        if (fd >= 0) ::close(fd);
    }
    File(const File &) = delete;
    File &operator=(const File &) = delete;

    // n bytes at absolute file position pos
    void read_abs(uint64_t pos, void *dst, uint64_t n) const
    {
        if (pos > size || n > size - pos) fail("'" + path + "': a structure reaches past the end of the file");
        uint8_t *d = static_cast<uint8_t *>(dst);
        while (n > 0) {
            const ssize_t r = ::pread(fd, d, n, (off_t)pos);
            if (r <= 0) fail("'" + path + "': read error");
            d += r;
            pos += (uint64_t)r;
            n -= (uint64_t)r;
        }
    }
    // n bytes at file address addr (relative to the base address)
    std::vector<uint8_t> read(uint64_t addr, uint64_t n) const
    {
        if (addr == kUndef) fail("'" + path + "': undefined address");
        if (addr > size || base > size - addr) fail("'" + path + "': address past the end of the file");
        const uint64_t pos = base + addr;
        if (n > size - pos) fail("'" + path + "': a structure reaches past the end of the file");
        std::vector<uint8_t> v(n);   // sized only after the range is known to lie in the file
        read_abs(pos, v.data(), n);
        return v;
    }
};

// little-endian field decoding with bounds checks on the buffer
struct Cursor {
    const std::vector<uint8_t> &b;
    size_t p;
    const File &f;
    Cursor(const std::vector<uint8_t> &buf, size_t pos, const File &file) : b(buf), p(pos), f(file) {}
    uint64_t uint(int n)
    {
        if (p + (size_t)n > b.size()) fail("'" + f.path + "': truncated header field");
        uint64_t v = 0;
        for (int i = 0; i < n; i++) v |= (uint64_t)b[p + i] << (8 * i);
        p += (size_t)n;
        return v;
    }
    uint64_t off() { return uint(f.so); }
    uint64_t len() { return uint(f.sl); }
    void skip(size_t n)
    {
        if (p + n > b.size()) fail("'" + f.path + "': truncated header field");
        p += n;
    }
};

struct Entry {   // symbol table entry
    uint64_t name_off = 0, header = kUndef;
    uint32_t cache = 0;
    uint64_t btree = kUndef, heap = kUndef;
};

Entry read_entry(Cursor &c)
{
    Entry e;
    e.name_off = c.off();
    e.header = c.off();
    e.cache = (uint32_t)c.uint(4);
    c.skip(4);
    const size_t scratch = c.p;
    if (e.cache == 1) {
        e.btree = c.off();
        e.heap = c.off();
    }
    c.p = scratch + 16;
    return e;
}

struct Message {
    uint16_t type;
    std::vector<uint8_t> data;
};

// The messages of a version-1 object header, continuation blocks followed.
std::vector<Message> object_messages(const File &f, uint64_t addr)
{
    const std::vector<uint8_t> pre = f.read(addr, 16);
    Cursor c(pre, 0, f);
    const int version = (int)c.uint(1);
    if (version != 1)
        fail("'" + f.path + "': object header version " + std::to_string(version) +
             " (only version 1 is read here)");
    c.skip(1);
    const uint64_t nmsg = c.uint(2);
    c.skip(4);   // reference count
    const uint64_t hsize = c.uint(4);
    std::vector<Message> out;
    std::vector<std::pair<uint64_t, uint64_t>> blocks{{addr + 16, hsize}};
    for (size_t k = 0; k < blocks.size() && out.size() < nmsg; k++) {
        if (blocks.size() > 1024) fail("'" + f.path + "': too many object header continuation blocks");
        const std::vector<uint8_t> blk = f.read(blocks[k].first, blocks[k].second);
        size_t p = 0;
        while (p + 8 <= blk.size() && out.size() < nmsg) {
            Cursor m(blk, p, f);
            const uint16_t type = (uint16_t)m.uint(2);
            const uint64_t sz = m.uint(2);
            m.skip(4);   // flags, reserved
            if (p + 8 + sz > blk.size()) fail("'" + f.path + "': object header message past its block");
            Message msg{type, std::vector<uint8_t>(blk.begin() + (long)(p + 8), blk.begin() + (long)(p + 8 + sz))};
            if (type == 0x10) {   // continuation: offset, length
                Cursor cc(msg.data, 0, f);
                const uint64_t a = cc.off(), l = cc.len();
                blocks.push_back({a, l});
            }
            out.push_back(std::move(msg));
            p += 8 + sz;
        }
    }
    return out;
}

std::string heap_name(const File &f, uint64_t heap_addr, uint64_t off)
{
    const std::vector<uint8_t> h = f.read(heap_addr, 32);
    if (std::memcmp(h.data(), "HEAP", 4) != 0) fail("'" + f.path + "': local heap signature missing");
    Cursor c(h, 8, f);
    const uint64_t dsize = c.len();
    c.len();   // free list head
    const uint64_t daddr = c.off();
    if (off >= dsize) fail("'" + f.path + "': link name offset outside the local heap");
    const uint64_t n = std::min<uint64_t>(dsize - off, 4096);
    const std::vector<uint8_t> s = f.read(daddr + off, n);
    const auto z = std::find(s.begin(), s.end(), (uint8_t)0);
    if (z == s.end()) fail("'" + f.path + "': unterminated link name");
    return std::string(s.begin(), z);
}

// Look name up among the links of the group whose symbol table is (btree, heap).
// A child node's level is one below its parent's (so no walk can cycle), and
// the walk visits at most kMaxNodes nodes (so no file can make it long).
constexpr int kMaxNodes = 1 << 16;

bool find_link(const File &f, uint64_t btree, uint64_t heap, const std::string &name, Entry &hit,
               int &visits, int expect_level = -1)
{
    if (++visits > kMaxNodes) fail("'" + f.path + "': group B-tree with more than 65536 nodes");
    const std::vector<uint8_t> hdr = f.read(btree, 8 + 2 * (uint64_t)f.so);
    if (std::memcmp(hdr.data(), "TREE", 4) != 0) fail("'" + f.path + "': B-tree node signature missing");
    if (hdr[4] != 0) fail("'" + f.path + "': not a group B-tree node");
    const int level = hdr[5];
    if (expect_level >= 0 && level != expect_level) fail("'" + f.path + "': B-tree child at the wrong level");
    const uint64_t nent = (uint64_t)hdr[6] | ((uint64_t)hdr[7] << 8);
    const uint64_t body = 8 + 2 * (uint64_t)f.so;
    const std::vector<uint8_t> node = f.read(btree, body + nent * (f.sl + f.so) + f.sl);
    Cursor c(node, body, f);
    for (uint64_t i = 0; i < nent; i++) {
        c.len();   // key: heap offset of the child's smallest name (not needed: every child is searched)
        const uint64_t child = c.off();
        if (level > 0) {
            if (find_link(f, child, heap, name, hit, visits, level - 1)) return true;
            continue;
        }
        const std::vector<uint8_t> sh = f.read(child, 8);
        if (std::memcmp(sh.data(), "SNOD", 4) != 0) fail("'" + f.path + "': symbol table node signature missing");
        const uint64_t nsym = (uint64_t)sh[6] | ((uint64_t)sh[7] << 8);
        const uint64_t esize = 2 * (uint64_t)f.so + 8 + 16;
        const std::vector<uint8_t> sn = f.read(child, 8 + nsym * esize);
        Cursor e(sn, 8, f);
        for (uint64_t k = 0; k < nsym; k++) {
            Entry en = read_entry(e);
            if (heap_name(f, heap, en.name_off) == name) {
                hit = en;
                return true;
            }
        }
    }
    return false;
}

// The symbol table (B-tree, heap) of the group at entry e.
void group_table(const File &f, const Entry &e, uint64_t &btree, uint64_t &heap)
{
    if (e.cache == 1 && e.btree != kUndef) {
        btree = e.btree;
        heap = e.heap;
        return;
    }
    for (const Message &m : object_messages(f, e.header)) {
        if (m.type == 0x11) {
            Cursor c(m.data, 0, f);
            btree = c.off();
            heap = c.off();
            return;
        }
    }
    fail("'" + f.path + "': a path element is not a group with a symbol table");
}

struct Dataset {
    std::vector<uint64_t> dims;
    int cls = -1, size = 0, big_endian = 0, is_signed = 0;
    int layout = -1;               // 0 compact, 1 contiguous
    uint64_t addr = kUndef, bytes = 0;
    std::vector<uint8_t> compact;
    uint64_t nelem() const   // checked against overflow when the dataset is opened
    {
        uint64_t n = 1;
        for (uint64_t d : dims) n *= d;
        return n;
    }
};

// The element count of dims, failing where it or its byte size exceeds 2^62
// (so that offsets and byte counts derived from it cannot wrap).
void check_extent(const File &f, const std::vector<uint64_t> &dims, int elem_size)
{
    constexpr uint64_t kMax = 1ull << 62;
    uint64_t n = 1;
    for (uint64_t d : dims) {
        if (d != 0 && n > kMax / d) fail("'" + f.path + "': dataspace too large");
        n *= d;
    }
    if (elem_size > 0 && n > kMax / (uint64_t)elem_size) fail("'" + f.path + "': dataspace too large");
}

Dataset open_dataset(File &f, const char *name)
{
    // superblock: signature at 0 or at 512 * 2^k
    static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    uint64_t at = 0;
    for (;;) {
        uint8_t s[8];
        if (at + 8 > f.size) fail("'" + f.path + "': not an HDF5 file (no superblock signature)");
        f.read_abs(at, s, 8);
        if (std::memcmp(s, sig, 8) == 0) break;
        at = at ? at * 2 : 512;
    }
    std::vector<uint8_t> sb(128);
    f.read_abs(at, sb.data(), std::min<uint64_t>(128, f.size - at));
    const int version = sb[8];
    if (version > 1)
        fail("'" + f.path + "': superblock version " + std::to_string(version) + " (only versions 0 and 1 are read here)");
    f.so = sb[13];
    f.sl = sb[14];
    if (f.so != 8 || f.sl != 8) fail("'" + f.path + "': offsets and lengths other than 8 bytes are not read here");
    Cursor c(sb, version == 0 ? 24 : 28, f);
    f.base = c.off();
    c.off();   // free-space info
    c.off();   // end of file
    c.off();   // driver information block
    const Entry root = read_entry(c);
    if (f.base != at && f.base != 0) fail("'" + f.path + "': unexpected base address");
    f.base = at;

    // walk the path
    Entry cur = root;
    std::string path = name;
    size_t p = 0;
    while (p < path.size()) {
        size_t q = path.find('/', p);
        if (q == std::string::npos) q = path.size();
        const std::string part = path.substr(p, q - p);
        p = q + 1;
        if (part.empty()) continue;
        uint64_t bt = kUndef, hp = kUndef;
        group_table(f, cur, bt, hp);
        Entry hit;
        int visits = 0;
        if (!find_link(f, bt, hp, part, hit, visits)) fail("'" + f.path + "': no dataset or group '" + part + "'");
        cur = hit;
    }

    Dataset d;
    bool have_space = false, have_type = false;
    for (const Message &m : object_messages(f, cur.header)) {
        Cursor mc(m.data, 0, f);
        switch (m.type) {
        case 0x01: {   // dataspace
            const int v = (int)mc.uint(1), rank = (int)mc.uint(1);
            mc.uint(1);   // flags
            int kind = 1;   // version 2: 0 scalar, 1 simple, 2 null
            if (v == 1) mc.skip(5);
            else if (v == 2) kind = (int)mc.uint(1);
            else fail("'" + f.path + "': dataspace message version " + std::to_string(v));
            if (rank > 32) fail("'" + f.path + "': dataspace rank above 32");
            for (int i = 0; i < rank; i++) d.dims.push_back(mc.len());
            if (kind == 2) d.dims.assign(1, 0);   // null dataspace: no elements
            have_space = true;
            break;
        }
        case 0x03: {   // datatype
            const uint64_t cv = mc.uint(1);
            const uint64_t bits = mc.uint(3);
            d.cls = (int)(cv & 15);
            d.size = (int)mc.uint(4);
            d.big_endian = (int)(bits & 1);
            d.is_signed = (int)((bits >> 3) & 1);
            if (d.cls == 1 && ((bits >> 6) & 1)) fail("'" + f.path + "': VAX floating-point order");
            have_type = true;
            break;
        }
        case 0x08: {   // data layout
            const int v = (int)mc.uint(1);
            if (v != 3 && v != 4) fail("'" + f.path + "': data layout message version " + std::to_string(v));
            d.layout = (int)mc.uint(1);
            if (d.layout == 0) {
                const uint64_t n = mc.uint(2);
                if (mc.p + n > m.data.size()) fail("'" + f.path + "': compact data past its message");
                d.compact.assign(m.data.begin() + (long)mc.p, m.data.begin() + (long)(mc.p + n));
                d.bytes = n;
            } else if (d.layout == 1) {
                d.addr = mc.off();
                d.bytes = mc.len();
            } else {
                fail("'" + f.path + "': chunked or virtual storage is not read here");
            }
            break;
        }
        case 0x0B:
            fail("'" + f.path + "': filtered (compressed) datasets are not read here");
        default:
            break;
        }
    }
    if (!have_space || !have_type || d.layout < 0) fail("'" + f.path + "': '" + path + "' is not a dataset");
    if (!((d.cls == 0 && (d.size == 1 || d.size == 2 || d.size == 4 || d.size == 8)) ||
          (d.cls == 1 && (d.size == 4 || d.size == 8))))
        fail("'" + f.path + "': datatype class " + std::to_string(d.cls) + " size " + std::to_string(d.size) +
             " is not read here");
    check_extent(f, d.dims, d.size);
    if (d.layout == 1 && d.addr != kUndef && d.bytes < d.nelem() * (uint64_t)d.size)
        fail("'" + f.path + "': contiguous storage smaller than the dataspace");
    return d;
}

template <class T>
void read_elems(File &f, const Dataset &d, uint64_t offset, uint64_t count, T *out)
{
    const uint64_t n = d.nelem();
    if (offset > n || count > n - offset) fail("'" + f.path + "': requested elements past the dataset's end");
    const uint64_t es = (uint64_t)d.size;
    std::vector<uint8_t> raw;
    if (d.layout == 0) {
        if ((offset + count) * es > d.compact.size()) fail("'" + f.path + "': compact data shorter than the dataspace");
        raw.assign(d.compact.begin() + (long)(offset * es), d.compact.begin() + (long)((offset + count) * es));
    } else if (d.addr == kUndef) {
        raw.assign(count * es, 0);   // never written: the fill value of an unset dataset is zero
    } else {
        raw = f.read(d.addr + offset * es, count * es);
    }
    for (uint64_t i = 0; i < count; i++) {
        uint8_t b[8];
        for (uint64_t k = 0; k < es; k++) b[k] = raw[i * es + (d.big_endian ? es - 1 - k : k)];
        uint64_t u = 0;
        for (uint64_t k = 0; k < es; k++) u |= (uint64_t)b[k] << (8 * k);
        if (d.cls == 1) {
            if (es == 8) {
                double v;
                std::memcpy(&v, &u, 8);
                out[i] = (T)v;
            } else {
                float v;
                const uint32_t u32 = (uint32_t)u;
                std::memcpy(&v, &u32, 4);
                out[i] = (T)v;
            }
        } else if (d.is_signed) {
            const int sh = (int)(64 - 8 * es);
            out[i] = (T)((int64_t)(u << sh) >> sh);
        } else {
            out[i] = (T)u;
        }
    }
}

}  // namespace

extern "C" {

int croma_b200_h5_shape(const char *path, const char *dataset, int *rank, long long *dims, int max_rank,
                        int *type_class, int *type_size)
{
    if (!path || !dataset) { set_error("h5_shape: null path or dataset"); return -1; }
    try {
        File f(path);
        const Dataset d = open_dataset(f, dataset);
        if (rank) *rank = (int)d.dims.size();
        if (dims)
            for (int i = 0; i < (int)d.dims.size() && i < max_rank; i++) dims[i] = (long long)d.dims[i];
        if (type_class) *type_class = d.cls;
        if (type_size) *type_size = d.size;
        return 0;
    } catch (const H5Error &e) {
        set_error(e.msg);
        return -1;
    }
}

int croma_b200_h5_read_f64(const char *path, const char *dataset, long long offset, long long count, double *out)
{
    if (!path || !dataset || offset < 0 || count < 0 || (count > 0 && !out)) {
        set_error("h5_read_f64: invalid arguments");
        return -1;
    }
    try {
        File f(path);
        const Dataset d = open_dataset(f, dataset);
        read_elems<double>(f, d, (uint64_t)offset, (uint64_t)count, out);
        return 0;
    } catch (const H5Error &e) {
        set_error(e.msg);
        return -1;
    }
}

int croma_b200_h5_read_i64(const char *path, const char *dataset, long long offset, long long count,
                           long long *out)
{
    if (!path || !dataset || offset < 0 || count < 0 || (count > 0 && !out)) {
        set_error("h5_read_i64: invalid arguments");
        return -1;
    }
    try {
        File f(path);
        const Dataset d = open_dataset(f, dataset);
        if (d.cls != 0) {
            set_error("h5_read_i64: '" + std::string(dataset) + "' is not an integer dataset");
            return -1;
        }
        read_elems<long long>(f, d, (uint64_t)offset, (uint64_t)count, out);
        return 0;
    } catch (const H5Error &e) {
        set_error(e.msg);
        return -1;
    }
}

}  // extern "C"
