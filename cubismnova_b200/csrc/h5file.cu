// HDF5 container files for grid data, written and read without the HDF5
// library (host code only).
//
// The reference hands its file buffer to libhdf5: one dataset "data" of
// dims (z, y, x, components) at the root of `fname.h5`, created with one
// chunk spanning the dataset (src/IO/HDFDriver.cpp:25-111), and reads it
// back as the hyperslab [0, count) (src/IO/HDFDriver.cpp:113-165).
// libhdf5 is not part of this build, so the file is laid out here from the
// published HDF5 file-format specification, in the structures libhdf5
// itself writes under its default (earliest) format bounds:
//
//   superblock version 0 (offsets and lengths of 8 bytes)
//   root group of the symbol-table kind: version 1 object header with a
//     symbol-table message -> v1 B-tree (group node, K = 16) -> one
//     symbol-table node (K = 4) whose entry names the dataset in the
//     group's local heap
//   dataset: version 1 object header with dataspace (v1), datatype (v1,
//     IEEE little-endian float or little-endian two's-complement integer),
//     fill value (v2) and data layout (v3) messages; the data contiguous,
//     or as one chunk indexed by a v1 B-tree (the reference's layout)
//
// The reader takes that subset wherever it appears: the superblock after
// a user block of 0, 512, 1024, ... bytes (versions 0 and 1), groups whose
// B-trees have any depth, v1 object headers with continuation blocks,
// dataspace messages of versions 1 and 2, data layout messages of versions
// 1 to 3 (compact, contiguous, chunked without filters), and it reads any
// hyperslab [0, count) of the dataset with conversion between FP64, FP32
// and INT32 values (integers to floats only).

#include "cn_internal.h"

#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace cn {
namespace h5 {

constexpr uint64_t kUndef = ~0ull;     // the undefined address
constexpr uint64_t kFreeNull = 1;      // end of a local heap's free list, as libhdf5 writes it
constexpr int kGroupLeafK = 4;         // symbol-table node: up to 2K entries
constexpr int kGroupInternalK = 16;    // group B-tree node: up to 2K children
constexpr int kChunkK = 32;            // chunk B-tree node (the default of a version 0 superblock)
constexpr int kEntrySize = 40;         // symbol-table entry with 8-byte offsets
constexpr int kMaxRank = 32;
const uint8_t kSignature[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};

enum Msg : uint16_t {
    kNil = 0x0000,
    kDataspace = 0x0001,
    kDatatype = 0x0003,
    kFillOld = 0x0004,
    kFill = 0x0005,
    kLayout = 0x0008,
    kFilters = 0x000B,
    kContinuation = 0x0010,
    kSymbolTable = 0x0011,
};

struct Writer {
    std::vector<uint8_t> b;
    size_t size() const { return b.size(); }
    void u8(uint64_t v) { b.push_back((uint8_t)v); }
    void le(uint64_t v, int n)
    {
        for (int i = 0; i < n; ++i) b.push_back((uint8_t)(v >> (8 * i)));
    }
    void u16(uint64_t v) { le(v, 2); }
    void u32(uint64_t v) { le(v, 4); }
    void u64(uint64_t v) { le(v, 8); }
    void bytes(const void *p, size_t n) { b.insert(b.end(), (const uint8_t *)p, (const uint8_t *)p + n); }
    void zeros(size_t n) { b.insert(b.end(), n, 0); }
    void pad_to(size_t pos) { zeros(pos > b.size() ? pos - b.size() : 0); }
};

struct TypeDesc {
    int cls;       // 0 fixed-point, 1 floating point
    uint32_t size; // bytes
    bool sgn;      // fixed-point: two's complement
};

inline bool type_of(cn_dtype t, TypeDesc &d)
{
    switch (t) {
    case CN_FLOAT64: d = {1, 8, true}; return true;
    case CN_FLOAT32: d = {1, 4, true}; return true;
    case CN_INT32: d = {0, 4, true}; return true;
    }
    return false;
}

// datatype message body, version 1 (class in the low nibble)
void put_datatype(Writer &w, const TypeDesc &t)
{
    if (t.cls == 1) {
        w.u8(0x10 | 1);
        w.u8(0x20); // little-endian, zero padding, mantissa normalised with an implied leading 1
        w.u8(t.size * 8 - 1); // sign bit position
        w.u8(0);
        w.u32(t.size);
        const bool dbl = t.size == 8;
        w.u16(0);                 // bit offset
        w.u16(t.size * 8);        // precision
        w.u8(dbl ? 52 : 23);      // exponent location
        w.u8(dbl ? 11 : 8);       // exponent size
        w.u8(0);                  // mantissa location
        w.u8(dbl ? 52 : 23);      // mantissa size
        w.u32(dbl ? 1023 : 127);  // exponent bias
    } else {
        w.u8(0x10 | 0);
        w.u8(t.sgn ? 0x08 : 0x00); // little-endian, zero padding, signed
        w.u8(0);
        w.u8(0);
        w.u32(t.size);
        w.u16(0);          // bit offset
        w.u16(t.size * 8); // precision
    }
}

// one message of a version 1 object header: 8-byte header, body padded to 8
void put_message(Writer &oh, uint16_t type, uint8_t flags, const Writer &body)
{
    const size_t n = (body.size() + 7) / 8 * 8;
    oh.u16(type);
    oh.u16(n);
    oh.u8(flags);
    oh.zeros(3);
    oh.bytes(body.b.data(), body.size());
    oh.zeros(n - body.size());
}

// version 1 object header: 16-byte prefix, then the messages
void put_object_header(Writer &f, int nmsgs, const Writer &msgs)
{
    f.u8(1);
    f.u8(0);
    f.u16(nmsgs);
    f.u32(1); // reference count
    f.u32(msgs.size());
    f.zeros(4);
    f.bytes(msgs.b.data(), msgs.size());
}

// Writes `path`: dataset `name` (root group) of the given dims and type, the
// values of `data` (row-major, last dim fastest).  chunked: one chunk over
// the dataset, indexed by a v1 B-tree (what the reference's H5Pset_chunk
// with the dataset dims gives); else contiguous.
cn_status write_file(const char *path, const char *name, int rank, const long long *dims, cn_dtype dtype,
                     const void *data, int chunked)
{
    TypeDesc t;
    if (!path || !name || !dims || rank < 1 || rank > kMaxRank || !type_of(dtype, t))
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_h5_write: path, dataset name, rank (1-32) or type invalid");
    const size_t nlen = strlen(name);
    if (nlen == 0 || strchr(name, '/'))
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_h5_write: the dataset name must be non-empty and hold no '/'");
    uint64_t count = 1;
    for (int i = 0; i < rank; ++i) {
        if (dims[i] < 0) return fail(CN_ERR_INVALID_ARGUMENT, "cn_h5_write: negative dimension");
        count *= (uint64_t)dims[i];
    }
    const uint64_t nbytes = count * t.size;
    if (nbytes && !data) return fail(CN_ERR_INVALID_ARGUMENT, "cn_h5_write: data is NULL");
    if (chunked) {
        for (int i = 0; i < rank; ++i)
            if (dims[i] < 1 || dims[i] > 0xffffffffll)
                return fail(CN_ERR_UNSUPPORTED, "cn_h5_write: a chunk dimension must be in [1, 2^32)");
        if (nbytes >= (1ull << 32))
            return fail(CN_ERR_UNSUPPORTED, "cn_h5_write: one chunk holds less than 4 GiB; write it contiguous");
    }

    // addresses (base address 0)
    const uint64_t A_ROOT = 96; // after the 96-byte superblock
    const uint64_t root_size = 16 + 8 + 16;
    const uint64_t A_HEAP = A_ROOT + root_size;
    const uint64_t name_off = 8;
    const uint64_t names_end = name_off + (nlen + 1 + 7) / 8 * 8;
    const uint64_t free_size = 16;
    const uint64_t heap_data = names_end + free_size;
    const uint64_t A_HEAPDATA = A_HEAP + 32;
    const uint64_t A_BTREE = A_HEAPDATA + heap_data;
    const uint64_t btree_size = 24 + 2 * kGroupInternalK * 8 + (2 * kGroupInternalK + 1) * 8;
    const uint64_t A_SNOD = A_BTREE + btree_size;
    const uint64_t snod_size = 8 + 2 * kGroupLeafK * kEntrySize;
    const uint64_t A_DSET = A_SNOD + snod_size;

    // dataset object header messages
    Writer msgs;
    int nmsgs = 0;
    {
        Writer m; // dataspace, version 1
        m.u8(1);
        m.u8(rank);
        m.u8(0); // no maximum dims
        m.zeros(5);
        for (int i = 0; i < rank; ++i) m.u64((uint64_t)dims[i]);
        put_message(msgs, kDataspace, 0, m);
        ++nmsgs;
    }
    {
        Writer m;
        put_datatype(m, t);
        put_message(msgs, kDatatype, 1, m);
        ++nmsgs;
    }
    {
        Writer m; // fill value, version 2: allocation late (contiguous) / incremental (chunked),
                  // written if set, no fill value defined
        m.u8(2);
        m.u8(chunked ? 3 : 2);
        m.u8(2);
        m.u8(0);
        put_message(msgs, kFill, 1, m);
        ++nmsgs;
    }
    // the layout message holds the data (or chunk index) address: placed
    // after the header, which has a fixed size by then
    const uint64_t layout_body = chunked ? 3 + 8 + 4 * (uint64_t)(rank + 1) : 18;
    const uint64_t dset_size = 16 + msgs.size() + 8 + (layout_body + 7) / 8 * 8;
    const uint64_t A_CHUNKTREE = A_DSET + dset_size;
    const uint64_t chunk_key = 8 + 8 * (uint64_t)(rank + 1);
    const uint64_t chunktree_size = chunked ? 24 + 2 * kChunkK * 8 + (2 * kChunkK + 1) * chunk_key : 0;
    const uint64_t A_DATA = (A_CHUNKTREE + chunktree_size + 7) / 8 * 8;
    const uint64_t eof = A_DATA + nbytes;
    {
        Writer m;
        m.u8(3);
        if (chunked) {
            m.u8(2);
            m.u8(rank + 1);
            m.u64(A_CHUNKTREE);
            for (int i = 0; i < rank; ++i) m.u32((uint32_t)dims[i]);
            m.u32(t.size);
        } else {
            m.u8(1);
            m.u64(nbytes ? A_DATA : kUndef);
            m.u64(nbytes);
        }
        put_message(msgs, kLayout, 0, m);
        ++nmsgs;
    }

    Writer f;
    // superblock, version 0
    f.bytes(kSignature, 8);
    f.u8(0); // superblock
    f.u8(0); // free-space storage
    f.u8(0); // root group symbol table entry
    f.u8(0);
    f.u8(0); // shared header message format
    f.u8(8); // size of offsets
    f.u8(8); // size of lengths
    f.u8(0);
    f.u16(kGroupLeafK);
    f.u16(kGroupInternalK);
    f.u32(0); // file consistency flags
    f.u64(0); // base address
    f.u64(kUndef); // free-space info
    f.u64(eof);
    f.u64(kUndef); // driver information block
    // root group symbol table entry (cache type 1: B-tree and heap addresses)
    f.u64(0);
    f.u64(A_ROOT);
    f.u32(1);
    f.u32(0);
    f.u64(A_BTREE);
    f.u64(A_HEAP);
    // root group object header: the symbol table message
    f.pad_to(A_ROOT);
    {
        Writer m, rm;
        m.u64(A_BTREE);
        m.u64(A_HEAP);
        put_message(rm, kSymbolTable, 0, m);
        put_object_header(f, 1, rm);
    }
    // local heap of the root group: "" at 0, the dataset name at 8, then
    // one free block to the end of the segment
    f.pad_to(A_HEAP);
    f.bytes("HEAP", 4);
    f.u8(0);
    f.zeros(3);
    f.u64(heap_data);
    f.u64(names_end); // head of the free list
    f.u64(A_HEAPDATA);
    f.zeros(8);
    f.bytes(name, nlen);
    f.pad_to(A_HEAPDATA + names_end);
    f.u64(kFreeNull);
    f.u64(free_size);
    // group B-tree: one leaf node over one symbol-table node
    f.pad_to(A_BTREE);
    f.bytes("TREE", 4);
    f.u8(0); // group node
    f.u8(0); // leaf level
    f.u16(1);
    f.u64(kUndef);
    f.u64(kUndef);
    f.u64(0);        // key: name offset of "" (below every name)
    f.u64(A_SNOD);   // child
    f.u64(name_off); // key: the child's largest name
    f.pad_to(A_BTREE + btree_size);
    // symbol-table node with the dataset's entry
    f.bytes("SNOD", 4);
    f.u8(1);
    f.u8(0);
    f.u16(1);
    f.u64(name_off);
    f.u64(A_DSET);
    f.u32(0); // nothing cached
    f.u32(0);
    f.zeros(16);
    f.pad_to(A_SNOD + snod_size);
    // dataset object header
    put_object_header(f, nmsgs, msgs);
    if (f.size() != A_DSET + dset_size) return fail(CN_ERR_INVALID_ARGUMENT, "cn_h5_write: internal layout error");
    if (chunked) {
        // chunk B-tree: one leaf entry; left key = (size, filter mask,
        // offset 0...), right key = offsets at the dataset's far corner
        f.bytes("TREE", 4);
        f.u8(1); // raw data chunks
        f.u8(0);
        f.u16(1);
        f.u64(kUndef);
        f.u64(kUndef);
        f.u32((uint32_t)nbytes);
        f.u32(0);
        for (int i = 0; i <= rank; ++i) f.u64(0);
        f.u64(A_DATA);
        f.u32(0);
        f.u32(0);
        for (int i = 0; i < rank; ++i) f.u64((uint64_t)dims[i]);
        f.u64(0);
        f.pad_to(A_CHUNKTREE + chunktree_size);
    }
    f.pad_to(A_DATA);

    FILE *fp = fopen(path, "wb");
    if (!fp) return fail(CN_ERR_FILE, std::string("cn_h5_write: can not create '") + path + "'");
    bool good = fwrite(f.b.data(), 1, f.size(), fp) == f.size();
    if (good && nbytes) good = fwrite(data, 1, nbytes, fp) == nbytes;
    good = (fclose(fp) == 0) && good;
    if (!good) return fail(CN_ERR_FILE, std::string("cn_h5_write: write to '") + path + "' failed");
    return ok();
}

// ---------------------------------------------------------------- reading

struct Reader {
    FILE *fp = nullptr;
    uint64_t fsize = 0, base = 0;
    std::string err;
    ~Reader()
    {
        if (fp) fclose(fp);
    }
    bool at(uint64_t abs, void *dst, uint64_t n)
    {
        if (abs > fsize || n > fsize - abs) {
            err = "reference beyond the end of the file";
            return false;
        }
        if (fseeko(fp, (off_t)abs, SEEK_SET) != 0 || fread(dst, 1, n, fp) != n) {
            err = "read failed";
            return false;
        }
        return true;
    }
    bool get(uint64_t addr, std::vector<uint8_t> &v, uint64_t n)
    {
        v.resize(n);
        return at(base + addr, v.data(), n);
    }
};

inline uint64_t rd(const uint8_t *p, int n)
{
    uint64_t v = 0;
    for (int i = 0; i < n; ++i) v |= (uint64_t)p[i] << (8 * i);
    return v;
}

struct Dataset {
    int rank = -1;
    uint64_t dims[kMaxRank];
    TypeDesc type{-1, 0, false};
    bool type_ok = false;
    int layout = -1; // 0 compact, 1 contiguous, 2 chunked
    uint64_t addr = kUndef, size = 0;
    std::vector<uint8_t> compact;
    int cdims = 0;
    uint64_t chunk[kMaxRank + 1];
    bool filtered = false;
};

struct Message {
    uint16_t type;
    std::vector<uint8_t> body;
};

// messages of a version 1 object header, continuation blocks followed
bool read_object_header(Reader &R, uint64_t addr, std::vector<Message> &out)
{
    std::vector<uint8_t> pre;
    if (!R.get(addr, pre, 16)) return false;
    if (pre[0] != 1) {
        R.err = "object header version " + std::to_string(pre[0]) + " (only version 1 is read)";
        return false;
    }
    const uint64_t nmsgs = rd(&pre[2], 2);
    std::vector<std::pair<uint64_t, uint64_t>> blocks{{addr + 16, rd(&pre[8], 4)}};
    for (size_t k = 0; k < blocks.size() && k < 4096; ++k) {
        std::vector<uint8_t> blk;
        if (!R.get(blocks[k].first, blk, blocks[k].second)) return false;
        size_t q = 0;
        while (q + 8 <= blk.size() && out.size() < nmsgs) {
            const uint16_t type = (uint16_t)rd(&blk[q], 2);
            const uint64_t sz = rd(&blk[q + 2], 2);
            if (q + 8 + sz > blk.size()) {
                R.err = "object header message beyond its block";
                return false;
            }
            if (blk[q + 4] & 0x02) {
                R.err = "shared object header messages are not read";
                return false;
            }
            Message m{type, std::vector<uint8_t>(blk.begin() + q + 8, blk.begin() + q + 8 + sz)};
            if (type == kContinuation && sz >= 16) blocks.push_back({rd(&m.body[0], 8), rd(&m.body[8], 8)});
            out.push_back(std::move(m));
            q += 8 + sz;
        }
    }
    return true;
}

bool parse_dataset(Reader &R, uint64_t addr, Dataset &D)
{
    std::vector<Message> msgs;
    if (!read_object_header(R, addr, msgs)) return false;
    for (const Message &m : msgs) {
        const std::vector<uint8_t> &b = m.body;
        if (m.type == kDataspace && b.size() >= 4) {
            const int ver = b[0];
            D.rank = b[1];
            const size_t off = ver == 1 ? 8 : 4;
            if ((ver != 1 && ver != 2) || D.rank > kMaxRank || b.size() < off + 8 * (size_t)D.rank) {
                R.err = "unsupported dataspace message";
                return false;
            }
            if (ver == 2 && b[3] == 2) D.rank = 0; // null dataspace
            for (int i = 0; i < D.rank; ++i) D.dims[i] = rd(&b[off + 8 * i], 8);
        } else if (m.type == kDatatype && b.size() >= 8) {
            const int cls = b[0] & 0x0f;
            const uint32_t size = (uint32_t)rd(&b[4], 4);
            const bool big_endian = b[1] & 0x01;
            D.type = {cls, size, (b[1] & 0x08) != 0};
            // floats: IEEE binary32 / binary64 (exponent and mantissa sizes), not VAX order
            const bool ieee = b.size() >= 20 && !(b[1] & 0x40) && b[13] == (size == 8 ? 11 : 8) &&
                              b[15] == (size == 8 ? 52 : 23);
            D.type_ok = !big_endian && ((cls == 1 && (size == 4 || size == 8) && ieee) ||
                                        (cls == 0 && (size == 1 || size == 2 || size == 4 || size == 8)));
        } else if (m.type == kLayout && b.size() >= 2) {
            const int ver = b[0];
            if (ver == 1 || ver == 2) {
                // version, dimensionality, class, 5 reserved, [address], dims (4 bytes each)
                const int nd = b[1];
                D.layout = b[2];
                size_t q = 8;
                if (D.layout != 0) D.addr = rd(&b[q], 8), q += 8;
                if (nd > kMaxRank + 1 || b.size() < q + 4 * (size_t)nd) {
                    R.err = "bad data layout message";
                    return false;
                }
                D.cdims = nd;
                uint64_t prod = 1;
                for (int i = 0; i < nd; ++i) D.chunk[i] = rd(&b[q + 4 * i], 4), prod *= D.chunk[i];
                q += 4 * (size_t)nd;
                if (D.layout == 0) {
                    const uint64_t n = b.size() >= q + 4 ? rd(&b[q], 4) : 0;
                    if (b.size() < q + 4 + n) {
                        R.err = "bad compact layout";
                        return false;
                    }
                    D.compact.assign(b.begin() + q + 4, b.begin() + q + 4 + n);
                } else if (D.layout == 1) {
                    D.size = prod;
                }
            } else if (ver == 3) {
                D.layout = b[1];
                if (D.layout == 0) {
                    const uint64_t n = rd(&b[2], 2);
                    if (b.size() < 4 + n) {
                        R.err = "bad compact layout";
                        return false;
                    }
                    D.compact.assign(b.begin() + 4, b.begin() + 4 + n);
                } else if (D.layout == 1) {
                    if (b.size() < 18) {
                        R.err = "bad contiguous layout";
                        return false;
                    }
                    D.addr = rd(&b[2], 8);
                    D.size = rd(&b[10], 8);
                } else if (D.layout == 2) {
                    const int nd = b[2];
                    if (nd < 1 || nd > kMaxRank + 1 || b.size() < 11 + 4 * (size_t)nd) {
                        R.err = "bad chunked layout";
                        return false;
                    }
                    D.addr = rd(&b[3], 8);
                    D.cdims = nd;
                    for (int i = 0; i < nd; ++i) D.chunk[i] = rd(&b[11 + 4 * i], 4);
                } else {
                    R.err = "unsupported data layout class";
                    return false;
                }
            } else {
                R.err = "data layout message version " + std::to_string(ver) + " (versions 1-3 are read)";
                return false;
            }
        } else if (m.type == kFilters) {
            D.filtered = true;
        }
    }
    if (D.rank < 0 || !D.type_ok || D.layout < 0) {
        R.err = D.rank < 0 || D.layout < 0 ? "not a dataset of a simple dataspace"
                                           : "datatype other than little-endian IEEE float or integer";
        return false;
    }
    return true;
}

// finds `name` among the entries of the group B-tree rooted at `node`
bool find_in_group(Reader &R, uint64_t node, const std::vector<uint8_t> &heap, const std::string &name,
                   uint64_t &ohdr, int depth = 0)
{
    if (depth > 64) {
        R.err = "group B-tree too deep";
        return false;
    }
    std::vector<uint8_t> h;
    if (!R.get(node, h, 24)) return false;
    if (memcmp(h.data(), "TREE", 4) != 0 || h[4] != 0) {
        R.err = "bad group B-tree node";
        return false;
    }
    const int level = h[5];
    const uint64_t used = rd(&h[6], 2);
    std::vector<uint8_t> kc;
    if (!R.get(node + 24, kc, used * 16 + 8)) return false;
    for (uint64_t i = 0; i < used; ++i) {
        const uint64_t child = rd(&kc[8 + 16 * i], 8);
        if (level > 0) {
            if (find_in_group(R, child, heap, name, ohdr, depth + 1)) return true;
            if (!R.err.empty()) return false;
            continue;
        }
        std::vector<uint8_t> s;
        if (!R.get(child, s, 8)) return false;
        if (memcmp(s.data(), "SNOD", 4) != 0) {
            R.err = "bad symbol-table node";
            return false;
        }
        const uint64_t n = rd(&s[6], 2);
        std::vector<uint8_t> ents;
        if (!R.get(child + 8, ents, n * kEntrySize)) return false;
        for (uint64_t e = 0; e < n; ++e) {
            const uint64_t off = rd(&ents[e * kEntrySize], 8);
            if (off >= heap.size()) continue;
            const char *p = (const char *)heap.data() + off;
            const size_t len = strnlen(p, heap.size() - off);
            if (name.size() == len && memcmp(p, name.data(), len) == 0) {
                ohdr = rd(&ents[e * kEntrySize + 8], 8);
                return true;
            }
        }
    }
    return false;
}

bool open_dataset(Reader &R, const char *path, const char *dname, Dataset &D)
{
    struct stat st;
    if (stat(path, &st) != 0 || !(R.fp = fopen(path, "rb"))) {
        R.err = "can not open the file";
        return false;
    }
    R.fsize = (uint64_t)st.st_size;
    // the superblock: at 0 or after a user block of 512 * 2^k bytes
    uint64_t sb = kUndef;
    for (uint64_t o = 0; o + 8 <= R.fsize; o = o ? 2 * o : 512) {
        uint8_t sig[8];
        if (!R.at(o, sig, 8)) return false;
        if (memcmp(sig, kSignature, 8) == 0) {
            sb = o;
            break;
        }
    }
    if (sb == kUndef) {
        R.err = "no HDF5 superblock";
        return false;
    }
    uint8_t s[100];
    if (!R.at(sb, s, std::min<uint64_t>(100, R.fsize - sb))) return false;
    const int ver = s[8];
    if (ver > 1) {
        R.err = "superblock version " + std::to_string(ver) + " (versions 0 and 1 are read)";
        return false;
    }
    if (s[13] != 8 || s[14] != 8) {
        R.err = "sizes of offsets and lengths other than 8";
        return false;
    }
    const size_t e = ver == 0 ? 24 : 28; // base address onwards
    R.base = rd(&s[e], 8);
    const uint8_t *root = &s[e + 32];
    const uint64_t root_oh = rd(root + 8, 8);
    // the root group's symbol table message
    std::vector<Message> msgs;
    if (!read_object_header(R, root_oh, msgs)) return false;
    uint64_t btree = kUndef, heap = kUndef;
    for (const Message &m : msgs)
        if (m.type == kSymbolTable && m.body.size() >= 16) btree = rd(&m.body[0], 8), heap = rd(&m.body[8], 8);
    if (btree == kUndef) {
        R.err = "root group without a symbol table (only old-style groups are read)";
        return false;
    }
    std::vector<uint8_t> hh, hd;
    if (!R.get(heap, hh, 32)) return false;
    if (memcmp(hh.data(), "HEAP", 4) != 0) {
        R.err = "bad local heap";
        return false;
    }
    if (!R.get(rd(&hh[24], 8), hd, rd(&hh[8], 8))) return false;
    std::string name(dname);
    while (!name.empty() && name[0] == '/') name.erase(0, 1);
    uint64_t oh = kUndef;
    if (!find_in_group(R, btree, hd, name, oh)) {
        if (R.err.empty()) R.err = "no dataset '" + name + "' in the root group";
        return false;
    }
    return parse_dataset(R, oh, D);
}

inline bool dtype_of(const TypeDesc &t, cn_dtype &d)
{
    if (t.cls == 1 && t.size == 8) return d = CN_FLOAT64, true;
    if (t.cls == 1 && t.size == 4) return d = CN_FLOAT32, true;
    if (t.cls == 0 && t.size == 4 && t.sgn) return d = CN_INT32, true;
    return false;
}

// one file value (little-endian, type t) as double / int64
inline double as_double(const uint8_t *p, const TypeDesc &t)
{
    if (t.cls == 1) {
        if (t.size == 8) {
            double v;
            memcpy(&v, p, 8);
            return v;
        }
        float v;
        memcpy(&v, p, 4);
        return v;
    }
    uint64_t u = rd(p, t.size);
    if (t.sgn && t.size < 8 && (u >> (8 * t.size - 1)) & 1) u |= ~0ull << (8 * t.size);
    return t.sgn ? (double)(int64_t)u : (double)u;
}

// copies n file values at src into dst of dtype out
bool convert(const uint8_t *src, const TypeDesc &t, uint64_t n, cn_dtype out, uint8_t *dst)
{
    cn_dtype same;
    if (dtype_of(t, same) && same == out) {
        memcpy(dst, src, n * t.size);
        return true;
    }
    if (out == CN_INT32) {
        if (t.cls != 0) return false; // floats to integers: not converted
        for (uint64_t i = 0; i < n; ++i) {
            const int32_t v = (int32_t)(int64_t)as_double(src + i * t.size, t);
            memcpy(dst + 4 * i, &v, 4);
        }
        return true;
    }
    for (uint64_t i = 0; i < n; ++i) {
        const double v = as_double(src + i * t.size, t);
        if (out == CN_FLOAT64)
            memcpy(dst + 8 * i, &v, 8);
        else {
            const float f = (float)v;
            memcpy(dst + 4 * i, &f, 4);
        }
    }
    return true;
}

// copies the part of a row-major block (origin org, extent ext, file type)
// inside the hyperslab [0, cnt) into out (extent cnt, type dt)
bool scatter_block(const uint8_t *blk, const uint64_t *org, const uint64_t *ext, int rank, const TypeDesc &t,
                   const uint64_t *cnt, cn_dtype dt, uint8_t *out, size_t osz)
{
    uint64_t lo[kMaxRank], hi[kMaxRank];
    for (int i = 0; i < rank; ++i) {
        lo[i] = org[i];
        hi[i] = std::min(org[i] + ext[i], cnt[i]);
        if (lo[i] >= hi[i]) return true;
    }
    // walk the rows of the last dimension
    uint64_t idx[kMaxRank];
    for (int i = 0; i < rank; ++i) idx[i] = lo[i];
    const uint64_t row = hi[rank - 1] - lo[rank - 1];
    while (true) {
        uint64_t so = 0, oo = 0;
        for (int i = 0; i < rank; ++i) {
            so = so * ext[i] + (idx[i] - org[i]);
            oo = oo * cnt[i] + idx[i];
        }
        if (!convert(blk + so * t.size, t, row, dt, out + oo * osz)) return false;
        int d = rank - 2;
        while (d >= 0 && ++idx[d] == hi[d]) idx[d] = lo[d], --d;
        if (d < 0) break;
    }
    return true;
}

bool read_chunks(Reader &R, const Dataset &D, uint64_t node, const uint64_t *cnt, cn_dtype dt, uint8_t *out,
                 size_t osz, int depth = 0)
{
    if (depth > 64) {
        R.err = "chunk B-tree too deep";
        return false;
    }
    const int nd = D.cdims; // rank + 1 (the last: the element)
    const uint64_t key = 8 + 8 * (uint64_t)nd;
    std::vector<uint8_t> h;
    if (!R.get(node, h, 24)) return false;
    if (memcmp(h.data(), "TREE", 4) != 0 || h[4] != 1) {
        R.err = "bad chunk B-tree node";
        return false;
    }
    const int level = h[5];
    const uint64_t used = rd(&h[6], 2);
    std::vector<uint8_t> kc;
    if (!R.get(node + 24, kc, used * (key + 8) + key)) return false;
    const int rank = nd - 1;
    uint64_t cbytes = D.type.size;
    for (int i = 0; i < rank; ++i) cbytes *= D.chunk[i];
    std::vector<uint8_t> buf;
    for (uint64_t i = 0; i < used; ++i) {
        const uint8_t *k = &kc[i * (key + 8)];
        const uint64_t child = rd(k + key, 8);
        if (level > 0) {
            if (!read_chunks(R, D, child, cnt, dt, out, osz, depth + 1)) return false;
            continue;
        }
        if (rd(k + 4, 4) != 0 || rd(k, 4) < cbytes) {
            R.err = "filtered or short chunk";
            return false;
        }
        uint64_t org[kMaxRank];
        bool touches = true;
        for (int d = 0; d < rank; ++d) {
            org[d] = rd(k + 8 + 8 * d, 8);
            touches = touches && org[d] < cnt[d];
        }
        if (!touches) continue;
        if (!R.get(child, buf, cbytes)) return false;
        if (!scatter_block(buf.data(), org, D.chunk, rank, D.type, cnt, dt, out, osz)) {
            R.err = "floating-point values are not converted to integers";
            return false;
        }
    }
    return true;
}

cn_status read_file(const char *path, const char *dname, int rank, const long long *count, cn_dtype dt, void *out)
{
    if (!path || !dname || !count || !out || rank < 1 || rank > kMaxRank || (dt != CN_FLOAT32 && dt != CN_FLOAT64 &&
                                                                             dt != CN_INT32))
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_h5_read: path, dataset, counts, buffer, rank or type invalid");
    Reader R;
    Dataset D;
    if (!open_dataset(R, path, dname, D))
        return fail(CN_ERR_FILE, std::string("cn_h5_read: '") + path + "': " + R.err);
    if (D.rank != rank) return fail(CN_ERR_SIZE_MISMATCH, "cn_h5_read: the dataset's rank differs");
    uint64_t cnt[kMaxRank], n = 1;
    for (int i = 0; i < rank; ++i) {
        if (count[i] < 0 || (uint64_t)count[i] > D.dims[i])
            return fail(CN_ERR_SIZE_MISMATCH, "cn_h5_read: the hyperslab [0, count) exceeds the dataset");
        cnt[i] = (uint64_t)count[i];
        n *= cnt[i];
    }
    if (n == 0) return ok();
    const size_t osz = dt == CN_FLOAT64 ? 8 : 4;
    if (D.filtered) return fail(CN_ERR_UNSUPPORTED, "cn_h5_read: filtered (compressed) datasets are not read");
    uint64_t total = D.type.size;
    for (int i = 0; i < rank; ++i) total *= D.dims[i];
    if (D.layout == 2) {
        if (D.cdims != rank + 1) return fail(CN_ERR_FILE, "cn_h5_read: chunk rank differs from the dataset's");
        if (D.addr == kUndef) {
            memset(out, 0, n * osz); // no chunk allocated: the default fill value
            return ok();
        }
        memset(out, 0, n * osz);
        if (!read_chunks(R, D, D.addr, cnt, dt, (uint8_t *)out, osz))
            return fail(CN_ERR_FILE, std::string("cn_h5_read: '") + path + "': " + R.err);
        return ok();
    }
    // contiguous or compact: the dataset in row-major order
    std::vector<uint8_t> all;
    const uint8_t *src = nullptr;
    if (D.layout == 0) {
        if (D.compact.size() < total) return fail(CN_ERR_FILE, "cn_h5_read: compact data shorter than the dataset");
        src = D.compact.data();
    } else {
        if (D.addr == kUndef) {
            memset(out, 0, n * osz);
            return ok();
        }
        if (D.size < total) return fail(CN_ERR_FILE, "cn_h5_read: contiguous storage shorter than the dataset");
        bool whole = true;
        for (int i = 0; i < rank; ++i) whole = whole && cnt[i] == D.dims[i];
        cn_dtype same;
        if (whole && dtype_of(D.type, same) && same == dt) { // straight into the caller's buffer
            if (!R.at(R.base + D.addr, out, total))
                return fail(CN_ERR_FILE, std::string("cn_h5_read: '") + path + "': " + R.err);
            return ok();
        }
        if (!R.get(D.addr, all, total)) return fail(CN_ERR_FILE, std::string("cn_h5_read: '") + path + "': " + R.err);
        src = all.data();
    }
    const uint64_t zero[kMaxRank] = {};
    if (!scatter_block(src, zero, D.dims, rank, D.type, cnt, dt, (uint8_t *)out, osz))
        return fail(CN_ERR_UNSUPPORTED, "cn_h5_read: floating-point values are not converted to integers");
    return ok();
}

} // namespace h5
} // namespace cn

extern "C" cn_status cn_h5_write(const char *path, const char *dataset, int rank, const long long *dims,
                                 cn_dtype dtype, const void *host_buf, int chunked)
{
    return cn::h5::write_file(path, dataset, rank, dims, dtype, host_buf, chunked);
}

extern "C" cn_status cn_h5_query(const char *path, const char *dataset, int *rank, long long dims[32],
                                 cn_dtype *dtype)
{
    if (!path || !dataset || !rank || !dims || !dtype)
        return cn::fail(CN_ERR_INVALID_ARGUMENT, "cn_h5_query: NULL argument");
    cn::h5::Reader R;
    cn::h5::Dataset D;
    if (!cn::h5::open_dataset(R, path, dataset, D))
        return cn::fail(CN_ERR_FILE, std::string("cn_h5_query: '") + path + "': " + R.err);
    cn_dtype t;
    if (!cn::h5::dtype_of(D.type, t))
        return cn::fail(CN_ERR_UNSUPPORTED, "cn_h5_query: the dataset's type is not FP64, FP32 or INT32");
    *rank = D.rank;
    for (int i = 0; i < D.rank; ++i) dims[i] = (long long)D.dims[i];
    *dtype = t;
    return cn::ok();
}

extern "C" cn_status cn_h5_read(const char *path, const char *dataset, int rank, const long long *count,
                                cn_dtype dtype, void *host_buf)
{
    return cn::h5::read_file(path, dataset, rank, count, dtype, host_buf);
}

// ------------------------------------------------- grids and XDMF wrappers

namespace cn {
namespace h5 {

inline std::string fmt_zyx(const double *v)
{
    char b[128];
    snprintf(b, sizeof b, "%.16g %.16g %.16g", v[2], v[1], v[0]);
    return b;
}

} // namespace h5
} // namespace cn

extern "C" cn_status cn_xdmf_write(const char *fname, const char *aname, cn_entity entity, const int begin[3],
                                   const int end[3], const double origin[3], const double h[3], int ncomp,
                                   cn_dtype file_dtype, double time, int format)
{
    using namespace cn;
    if (!fname || !aname || !begin || !end || !origin || !h || ncomp < 1 || (format != 0 && format != 1))
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_xdmf_write: NULL argument, ncomp < 1 or unknown format");
    if (entity != CN_ENTITY_CELL && entity != CN_ENTITY_NODE)
        return fail(CN_ERR_UNSUPPORTED, "cn_xdmf_write: cell or node data only (face data gets no XDMF wrapper)");
    if (file_dtype != CN_FLOAT32 && file_dtype != CN_FLOAT64 && file_dtype != CN_INT32)
        return fail(CN_ERR_INVALID_ARGUMENT, "cn_xdmf_write: unknown file type");
    const bool node = entity == CN_ENTITY_NODE;
    int ext[3];
    double mesh_nodes[3], org[3];
    for (int d = 0; d < 3; ++d) {
        ext[d] = end[d] - begin[d];
        if (ext[d] < 0) return fail(CN_ERR_INVALID_ARGUMENT, "cn_xdmf_write: file range end before begin");
        // the mesh of the range: its cells (nodes minus one for node data)
        mesh_nodes[d] = node ? ext[d] : ext[d] + 1;
        org[d] = origin[d] + begin[d] * h[d];
    }
    const std::string path = std::string(fname) + ".xmf";
    FILE *x = fopen(path.c_str(), "w");
    if (!x) return fail(CN_ERR_FILE, "cn_xdmf_write: can not create '" + path + "'");
    const char *attr = ncomp == 1 ? "Scalar" : (ncomp == 3 ? "Vector" : "Tensor");
    std::string base(fname);
    base = base.substr(base.find_last_of('/') + 1);
    const int prec = file_dtype == CN_FLOAT64 ? 8 : 4;
    fprintf(x, "<?xml version=\"1.0\" ?>\n");
    fprintf(x, "<!DOCTYPE Xdmf SYSTEM \"Xdmf.dtd\" []>\n");
    fprintf(x, "<Xdmf Version=\"2.0\">\n");
    fprintf(x, "<Domain>\n");
    fprintf(x, "\t<Grid GridType=\"Uniform\">\n");
    fprintf(x, "\t\t<Time Value=\"%e\"/>\n\n", time);
    fprintf(x, "\t\t<Topology TopologyType=\"3DCoRectMesh\" Dimensions=\"%d %d %d\"/>\n\n", (int)mesh_nodes[2],
            (int)mesh_nodes[1], (int)mesh_nodes[0]);
    fprintf(x, "\t\t<Geometry GeometryType=\"Origin_DxDyDz\">\n");
    fprintf(x, "\t\t\t<DataItem Name=\"Origin\" Dimensions=\"3\" NumberType=\"Float\" Precision=\"8\" "
               "Format=\"XML\">\n");
    fprintf(x, "\t\t\t\t%s\n", h5::fmt_zyx(org).c_str());
    fprintf(x, "\t\t\t</DataItem>\n");
    fprintf(x, "\t\t\t<DataItem Name=\"Spacing\" Dimensions=\"3\" NumberType=\"Float\" Precision=\"8\" "
               "Format=\"XML\">\n");
    fprintf(x, "\t\t\t\t%s\n", h5::fmt_zyx(h).c_str());
    fprintf(x, "\t\t\t</DataItem>\n");
    fprintf(x, "\t\t</Geometry>\n\n");
    fprintf(x, "\t\t<Attribute Name=\"%s\" AttributeType=\"%s\" Center=\"%s\">\n", aname, attr,
            node ? "Node" : "Cell");
    if (format == 0) {
        fprintf(x, "\t\t\t<DataItem Dimensions=\"%d %d %d %d\" NumberType=\"%s\" Precision=\"%d\" Format=\"HDF\">\n",
                ext[2], ext[1], ext[0], ncomp, file_dtype == CN_INT32 ? "Int" : "Float", prec);
        fprintf(x, "\t\t\t\t./%s.h5:/data\n", base.c_str());
    } else {
        fprintf(x, "\t\t\t<DataItem Dimensions=\"%d %d %d %d\" NumberType=\"%s\" Precision=\"%d\" "
                   "Format=\"Binary\" Endian=\"Little\">\n",
                ext[2], ext[1], ext[0], ncomp, file_dtype == CN_INT32 ? "Int" : "Float", prec);
        fprintf(x, "\t\t\t\t./%s.bin\n", base.c_str());
    }
    fprintf(x, "\t\t\t</DataItem>\n");
    fprintf(x, "\t\t</Attribute>\n");
    fprintf(x, "\t</Grid>\n");
    fprintf(x, "</Domain>\n");
    fprintf(x, "</Xdmf>\n");
    if (fclose(x) != 0) return fail(CN_ERR_FILE, "cn_xdmf_write: write to '" + path + "' failed");
    return ok();
}

namespace {

struct HostBuf {
    void *p = nullptr;
    ~HostBuf() { free(p); }
};
struct DevBuf {
    void *p = nullptr;
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
};

// checks a file range and gives the dataset dims (z, y, x, ncomp) and bytes
cn_status file_dims(const cn_grid *g, int comp0, int *ncomp, const int b[3], const int e[3], cn_dtype fdt,
                    long long dims[4], size_t &bytes, const char *who)
{
    using namespace cn;
    if (!g || !b || !e) return fail(CN_ERR_INVALID_ARGUMENT, std::string(who) + ": grid or file range is NULL");
    if (*ncomp < 0) *ncomp = g->ncomp - comp0;
    if (comp0 < 0 || *ncomp < 1 || comp0 + *ncomp > g->ncomp)
        return fail(CN_ERR_INVALID_ARGUMENT, std::string(who) + ": components out of range");
    if (fdt != CN_FLOAT32 && fdt != CN_FLOAT64 && fdt != CN_INT32)
        return fail(CN_ERR_INVALID_ARGUMENT, std::string(who) + ": unknown file type");
    size_t n = (size_t)*ncomp;
    for (int d = 0; d < 3; ++d) {
        if (e[d] < b[d]) return fail(CN_ERR_INVALID_ARGUMENT, std::string(who) + ": file range end before begin");
        dims[2 - d] = e[d] - b[d];
        n *= (size_t)(e[d] - b[d]);
    }
    dims[3] = *ncomp;
    bytes = n * (fdt == CN_FLOAT64 ? 8 : 4);
    return ok();
}

} // namespace

extern "C" cn_status cn_grid_write_hdf(cn_grid *g, const char *fname, const char *aname, int comp0, int ncomp,
                                       const int begin[3], const int end[3], cn_dtype file_dtype, double time,
                                       int create_xdmf, void *stream)
{
    using namespace cn;
    if (!fname || !aname) return fail(CN_ERR_INVALID_ARGUMENT, "cn_grid_write_hdf: file or quantity name is NULL");
    long long dims[4];
    size_t bytes = 0;
    cn_status st = file_dims(g, comp0, &ncomp, begin, end, file_dtype, dims, bytes, "cn_grid_write_hdf");
    if (st != CN_OK) return st;
    if (create_xdmf) {
        printf("CartesianWriteHDF: Allocating %.1f MB file buffer (%s)\n", bytes / 1024. / 1024., fname);
        fflush(stdout);
    }
    HostBuf host;
    DevBuf dev;
    if (bytes) {
        if (!(host.p = malloc(bytes))) return fail(CN_ERR_OUT_OF_MEMORY, "cn_grid_write_hdf: host file buffer");
        CN_CUDA_TRY(cudaMalloc(&dev.p, bytes));
        cudaStream_t s = (cudaStream_t)stream;
        st = cn_grid_to_aos(g, comp0, ncomp, begin, end, file_dtype, dev.p, stream);
        if (st != CN_OK) return st;
        CN_CUDA_TRY(cudaMemcpyAsync(host.p, dev.p, bytes, cudaMemcpyDeviceToHost, s));
        CN_CUDA_TRY(cudaStreamSynchronize(s));
    }
    st = h5::write_file((std::string(fname) + ".h5").c_str(), "data", 4, dims, file_dtype, host.p, 0);
    if (st != CN_OK) return st;
    if (create_xdmf && (g->entity == CN_ENTITY_CELL || g->entity == CN_ENTITY_NODE))
        return cn_xdmf_write(fname, aname, (cn_entity)g->entity, begin, end, g->begin, g->h, ncomp, file_dtype, time,
                             0);
    return ok();
}

extern "C" cn_status cn_grid_read_hdf(cn_grid *g, const char *fname, int comp0, int ncomp, const int begin[3],
                                      const int end[3], cn_dtype file_dtype, void *stream)
{
    using namespace cn;
    if (!fname) return fail(CN_ERR_INVALID_ARGUMENT, "cn_grid_read_hdf: file name is NULL");
    const std::string path = std::string(fname) + ".h5";
    {
        FILE *f = fopen(path.c_str(), "rb");
        if (!f) return fail(CN_ERR_FILE, std::string("CartesianReadHDF: File '") + fname + "' does not exist");
        fclose(f);
    }
    long long dims[4];
    size_t bytes = 0;
    cn_status st = file_dims(g, comp0, &ncomp, begin, end, file_dtype, dims, bytes, "cn_grid_read_hdf");
    if (st != CN_OK || bytes == 0) return st;
    HostBuf host;
    DevBuf dev;
    if (!(host.p = malloc(bytes))) return fail(CN_ERR_OUT_OF_MEMORY, "cn_grid_read_hdf: host file buffer");
    st = h5::read_file(path.c_str(), "data", 4, dims, file_dtype, host.p);
    if (st != CN_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    CN_CUDA_TRY(cudaMalloc(&dev.p, bytes));
    CN_CUDA_TRY(cudaMemcpyAsync(dev.p, host.p, bytes, cudaMemcpyHostToDevice, s));
    st = cn_grid_from_aos(g, comp0, ncomp, begin, end, file_dtype, dev.p, stream);
    if (st != CN_OK) return st;
    // the buffers are released on return: wait for the scatter
    CN_CUDA_TRY(cudaStreamSynchronize(s));
    return ok();
}
