// spk_hdf5.hpp -- the snapshot files of the reference (src/io/hdf5_io.cu:19-252):
// HDF5 files holding 1-element datasets t_start, t_save, t_lastsnap,
// t_lastvar (f8) and step (i4), and one 1-D dataset of NX*NY*NZ f8 per field
// (named vx vy vz bx by bz th), the real field in C order (x slowest).
//
// The reference writes them through HighFive/libhdf5 with default property
// lists, which produce the original file format: superblock version 0, a
// root group indexed by a version-1 B-tree of symbol-table nodes with its
// names in a local heap, version-1 object headers, contiguous datasets.  No
// HDF5 library is available here, so this file writes and reads that format
// directly, following the HDF5 File Format Specification (superblock v0,
// "TREE" v1 B-tree node type 0, "SNOD" symbol table node, "HEAP" local heap,
// object header v1 with Dataspace 0x0001, Datatype 0x0003, Data Layout 0x0008
// (version 3) and Symbol Table 0x0011 messages).  The reader accepts the same
// format as written by libhdf5's defaults (for example h5py's initial
// conditions in the reference's tests): any number of symbol-table nodes and
// B-tree levels, continuation messages, unknown messages skipped, contiguous
// or compact layout, fixed-point and IEEE floating-point data of either byte
// order.  Host code only.
#pragma once
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace spkh5 {

enum DType { F64 = 0, I32 = 1 };

struct Dataset {
    std::string name;
    DType type = F64;
    std::vector<double> f64;    // F64 data
    std::vector<int32_t> i32;   // I32 data
    size_t size() const { return type == F64 ? f64.size() : i32.size(); }
};

static const uint64_t UNDEF = ~(uint64_t)0;
// end of a local heap's free list as libhdf5 stores it on disk
static const uint64_t HEAP_FREE_NULL = 1;
static const int LEAF_K = 8;        // symbol table node: up to 2K entries
static const int INTERNAL_K = 16;   // group B-tree node: up to 2K children
static const size_t ENTRY = 40;     // symbol table entry with 8-byte offsets

// ---- little-endian byte buffer -----------------------------------------------
struct Buf {
    std::vector<uint8_t> b;
    size_t size() const { return b.size(); }
    void u8(unsigned v) { b.push_back((uint8_t)v); }
    void u16(unsigned v) { for (int i = 0; i < 2; i++) b.push_back((uint8_t)(v >> (8 * i))); }
    void u32(uint32_t v) { for (int i = 0; i < 4; i++) b.push_back((uint8_t)(v >> (8 * i))); }
    void u64(uint64_t v) { for (int i = 0; i < 8; i++) b.push_back((uint8_t)(v >> (8 * i))); }
    void bytes(const void* p, size_t n) { b.insert(b.end(), (const uint8_t*)p, (const uint8_t*)p + n); }
    void zeros(size_t n) { b.insert(b.end(), n, 0); }
    void align8() { while (b.size() % 8) b.push_back(0); }
    void put64(size_t at, uint64_t v) { for (int i = 0; i < 8; i++) b[at + i] = (uint8_t)(v >> (8 * i)); }
};

static size_t pad8(size_t n) { return (n + 7) & ~(size_t)7; }

// One version-1 object header message: type, data size (a multiple of 8),
// flags, three reserved bytes, data.
static void message(Buf& o, unsigned type, const Buf& data) {
    const size_t n = pad8(data.size());
    o.u16(type);
    o.u16((unsigned)n);
    o.u8(0);
    o.zeros(3);
    o.bytes(data.b.data(), data.size());
    o.zeros(n - data.size());
}

// Version-1 object header: version 1, reserved, message count, reference
// count 1, chunk size, 4 bytes of padding to the 8-byte aligned messages.
static void object_header(Buf& o, int nmsg, const Buf& msgs) {
    o.u8(1);
    o.u8(0);
    o.u16((unsigned)nmsg);
    o.u32(1);
    o.u32((uint32_t)msgs.size());
    o.u32(0);
    o.bytes(msgs.b.data(), msgs.size());
}

// Writes the datasets into one file (names sorted as HDF5 requires for the
// symbol-table index); returns false with *why set on failure.
inline bool write_file(const std::string& path, std::vector<Dataset> ds, std::string* why) {
    std::sort(ds.begin(), ds.end(), [](const Dataset& a, const Dataset& b) { return strcmp(a.name.c_str(), b.name.c_str()) < 0; });
    for (size_t i = 0; i < ds.size(); i++) {
        if (ds[i].name.empty() || (i && ds[i].name == ds[i - 1].name)) { *why = "empty or repeated dataset name"; return false; }
    }
    const size_t nds = ds.size();
    const size_t per_node = 2 * LEAF_K;
    const size_t nsnod = nds ? (nds + per_node - 1) / per_node : 1;
    if (nsnod > 2 * (size_t)INTERNAL_K) { *why = "too many datasets for one B-tree node"; return false; }

    // local heap data segment: "" at offset 0, then the names
    Buf heap;
    heap.zeros(8);
    std::vector<uint64_t> name_off(nds);
    for (size_t i = 0; i < nds; i++) {
        name_off[i] = heap.size();
        heap.bytes(ds[i].name.c_str(), ds[i].name.size() + 1);
        heap.align8();
    }

    // addresses
    const size_t SB = 96;
    Buf root_msgs;                       // symbol table message: B-tree, heap (filled below)
    const size_t root_oh = SB;
    const size_t root_size = 16 + 8 + 16;
    const size_t heap_hdr = root_oh + root_size;
    const size_t heap_data = heap_hdr + 32;
    const size_t btree = heap_data + heap.size();
    const size_t btree_size = 24 + 2 * INTERNAL_K * 8 + (2 * INTERNAL_K + 1) * 8;
    const size_t snod0 = btree + btree_size;
    const size_t snod_size = 8 + per_node * ENTRY;
    size_t at = snod0 + nsnod * snod_size;
    std::vector<size_t> oh_addr(nds), data_addr(nds), data_bytes(nds);
    std::vector<Buf> oh(nds);
    for (size_t i = 0; i < nds; i++) {
        const Dataset& d = ds[i];
        data_bytes[i] = d.size() * (d.type == F64 ? 8 : 4);
        Buf msgs;
        Buf space;                       // dataspace v1: rank 1, no maximum dims
        space.u8(1); space.u8(1); space.u8(0); space.u8(0); space.u32(0);
        space.u64(d.size());
        message(msgs, 0x0001, space);
        Buf type;                        // datatype v1
        if (d.type == F64) {
            type.u8(0x11);               // version 1, class 1 (floating point)
            type.u8(0x20); type.u8(63); type.u8(0);   // LE, implied mantissa MSB, sign at bit 63
            type.u32(8);
            type.u16(0); type.u16(64);   // bit offset, precision
            type.u8(52); type.u8(11);    // exponent location, size
            type.u8(0); type.u8(52);     // mantissa location, size
            type.u32(1023);              // exponent bias
        } else {
            type.u8(0x10);               // version 1, class 0 (fixed point)
            type.u8(0x08); type.u8(0); type.u8(0);    // LE, signed
            type.u32(4);
            type.u16(0); type.u16(32);
        }
        message(msgs, 0x0003, type);
        oh[i] = msgs;                    // layout message appended once the address is known
        oh_addr[i] = at;
        at += 16 + msgs.size() + 8 + 24;
    }
    for (size_t i = 0; i < nds; i++) {
        at = pad8(at);
        data_addr[i] = at;
        at += data_bytes[i];
    }
    const size_t eof = pad8(at);

    Buf f;
    // superblock version 0
    const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    f.bytes(sig, 8);
    f.u8(0); f.u8(0); f.u8(0); f.u8(0);  // superblock, free-space, root entry versions, reserved
    f.u8(0); f.u8(8); f.u8(8); f.u8(0);  // shared header version, size of offsets, of lengths, reserved
    f.u16(LEAF_K); f.u16(INTERNAL_K);
    f.u32(0);                            // consistency flags
    f.u64(0);                            // base address
    f.u64(UNDEF);                        // free-space info
    f.u64(eof);                          // end of file address
    f.u64(UNDEF);                        // driver information block
    // root group symbol table entry (scratch pad caches the B-tree and heap)
    f.u64(0); f.u64(root_oh); f.u32(1); f.u32(0); f.u64(btree); f.u64(heap_hdr);
    // root object header: one symbol table message
    Buf stab;
    stab.u64(btree); stab.u64(heap_hdr);
    message(root_msgs, 0x0011, stab);
    object_header(f, 1, root_msgs);
    // local heap
    f.bytes("HEAP", 4); f.u8(0); f.zeros(3);
    f.u64(heap.size()); f.u64(HEAP_FREE_NULL); f.u64(heap_data);
    f.bytes(heap.b.data(), heap.size());
    // B-tree node, type 0 (group), level 0: children are the symbol table nodes
    f.bytes("TREE", 4); f.u8(0); f.u8(0); f.u16((unsigned)nsnod);
    f.u64(UNDEF); f.u64(UNDEF);
    f.u64(0);                            // key 0: the empty name
    for (size_t s = 0; s < nsnod; s++) {
        f.u64(snod0 + s * snod_size);
        const size_t last = std::min(nds, (s + 1) * per_node);
        f.u64(nds ? name_off[last - 1] : 0);   // key s+1: the greatest name of child s
    }
    f.zeros(btree_size - (24 + 8 + nsnod * 16));
    // symbol table nodes
    for (size_t s = 0; s < nsnod; s++) {
        const size_t first = s * per_node, last = std::min(nds, first + per_node);
        f.bytes("SNOD", 4); f.u8(1); f.u8(0); f.u16((unsigned)(last - first));
        for (size_t i = first; i < last; i++) {
            f.u64(name_off[i]); f.u64(oh_addr[i]); f.u32(0); f.u32(0); f.zeros(16);
        }
        f.zeros((per_node - (last - first)) * ENTRY);
    }
    // dataset object headers
    for (size_t i = 0; i < nds; i++) {
        if (f.size() != oh_addr[i]) { *why = "internal layout error"; return false; }
        Buf lay;                         // data layout v3, contiguous
        lay.u8(3); lay.u8(1); lay.u64(data_addr[i]); lay.u64(data_bytes[i]);
        Buf msgs = oh[i];
        message(msgs, 0x0008, lay);
        object_header(f, 3, msgs);
    }
    // raw data
    for (size_t i = 0; i < nds; i++) {
        while (f.size() < data_addr[i]) f.u8(0);
        if (ds[i].type == F64) {
            for (double v : ds[i].f64) { uint64_t u; memcpy(&u, &v, 8); f.u64(u); }
        } else {
            for (int32_t v : ds[i].i32) f.u32((uint32_t)v);
        }
    }
    while (f.size() < eof) f.u8(0);

    FILE* fp = fopen(path.c_str(), "wb");
    if (!fp) { *why = "cannot create " + path; return false; }
    const bool ok = fwrite(f.b.data(), 1, f.size(), fp) == f.size();
    if (fclose(fp) != 0 || !ok) { *why = "cannot write " + path; return false; }
    return true;
}

// ---- reader --------------------------------------------------------------------
class Reader {
public:
    bool open(const std::string& path, std::string* why) {
        FILE* fp = fopen(path.c_str(), "rb");
        if (!fp) { *why = "cannot open " + path; return false; }
        fseek(fp, 0, SEEK_END);
        const long n = ftell(fp);
        fseek(fp, 0, SEEK_SET);
        d_.resize(n > 0 ? (size_t)n : 0);
        const bool ok = n > 0 && fread(d_.data(), 1, d_.size(), fp) == d_.size();
        fclose(fp);
        if (!ok) { *why = "cannot read " + path; return false; }
        return parse(why);
    }
    // names and object header addresses of the root group
    const std::vector<std::pair<std::string, uint64_t>>& entries() const { return ent_; }

    // Reads dataset `name` (any shape; flattened) converted to doubles or
    // int32s; false with *why when it is missing or not readable.
    bool read(const std::string& name, DType want, Dataset* out, std::string* why) {
        uint64_t oh = UNDEF;
        for (auto& e : ent_) if (e.first == name) oh = e.second;
        if (oh == UNDEF) { *why = "no dataset " + name; return false; }
        Info info;
        if (!object(oh, &info, why)) { *why = name + ": " + *why; return false; }
        if (!info.have_space || !info.have_type || !info.have_layout) { *why = name + ": not a dataset"; return false; }
        const size_t n = info.nelem, es = info.esize;
        const uint8_t* src = nullptr;
        if (info.compact) src = info.compact_data.data();
        else {
            if (info.addr == UNDEF) { *why = name + ": data not allocated"; return false; }
            if (!in(info.addr, n * es)) { *why = name + ": data beyond the end of the file"; return false; }
            src = d_.data() + base_ + info.addr;
        }
        if (info.compact && info.compact_data.size() < n * es) { *why = name + ": short compact data"; return false; }
        out->name = name;
        out->type = want;
        out->f64.clear();
        out->i32.clear();
        for (size_t i = 0; i < n; i++) {
            uint8_t v[8];
            for (size_t b = 0; b < es; b++) v[b] = src[i * es + (info.big_endian ? es - 1 - b : b)];
            double x;
            if (info.cls == 1) {
                if (es == 8) { memcpy(&x, v, 8); }
                else { float y; memcpy(&y, v, 4); x = y; }
            } else {
                int64_t iv = 0;
                for (size_t b = 0; b < es; b++) iv |= (int64_t)v[b] << (8 * b);
                if (info.is_signed && es < 8 && (v[es - 1] & 0x80)) iv -= (int64_t)1 << (8 * es);
                x = info.is_signed ? (double)iv : (double)(uint64_t)iv;
            }
            if (want == F64) out->f64.push_back(x);
            else out->i32.push_back((int32_t)x);
        }
        return true;
    }

private:
    std::vector<uint8_t> d_;
    uint64_t base_ = 0;
    int so_ = 8, sl_ = 8;
    std::vector<std::pair<std::string, uint64_t>> ent_;

    struct Info {
        bool have_space = false, have_type = false, have_layout = false;
        size_t nelem = 0, esize = 0;
        int cls = -1;
        bool big_endian = false, is_signed = false;
        bool compact = false;
        uint64_t addr = UNDEF;
        std::vector<uint8_t> compact_data;
        uint64_t stab_btree = UNDEF, stab_heap = UNDEF;
    };

    bool in(uint64_t a, uint64_t n) const { return a != UNDEF && base_ + a <= d_.size() && n <= d_.size() - (base_ + a); }
    uint64_t get(uint64_t a, int n) const {
        uint64_t v = 0;
        for (int i = 0; i < n; i++) v |= (uint64_t)d_[base_ + a + i] << (8 * i);
        if (n < 8 && v == ((uint64_t)1 << (8 * n)) - 1) return UNDEF;
        return v;
    }
    uint64_t raw(uint64_t a, int n) const {   // no undefined-address mapping
        uint64_t v = 0;
        for (int i = 0; i < n; i++) v |= (uint64_t)d_[base_ + a + i] << (8 * i);
        return v;
    }

    bool parse(std::string* why) {
        static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
        // the signature may sit at 0, 512, 1024, ... (a user block before it)
        size_t at = 0;
        while (at + 8 <= d_.size() && memcmp(d_.data() + at, sig, 8) != 0) at = at ? at * 2 : 512;
        if (at + 8 > d_.size()) { *why = "not an HDF5 file (no signature)"; return false; }
        const uint8_t ver = d_[at + 8];
        if (ver > 1) { *why = "superblock version " + std::to_string(ver) + " is not supported (0 and 1 are)"; return false; }
        so_ = d_[at + 13];
        sl_ = d_[at + 14];
        if (so_ != 8 || sl_ != 8) { *why = "only 8-byte offsets and lengths are supported"; return false; }
        // superblock fields at absolute positions, then addresses relative to the base
        size_t p = at + 24 + (ver == 1 ? 4 : 0);
        base_ = 0;
        if (p + 4 * 8 + ENTRY > d_.size()) { *why = "truncated superblock"; return false; }
        const uint64_t base = raw(p, 8);
        p += 4 * 8;                       // base, free space, end of file, driver block
        const uint64_t root_oh = raw(p + 8, 8);
        const uint32_t cache = (uint32_t)raw(p + 16, 4);
        uint64_t btree = UNDEF, heap = UNDEF;
        if (cache == 1) { btree = raw(p + 24, 8); heap = raw(p + 32, 8); }
        base_ = base == UNDEF ? at : base;
        if (cache != 1) {
            Info ri;
            if (!object(root_oh, &ri, why)) return false;
            btree = ri.stab_btree; heap = ri.stab_heap;
        }
        if (btree == UNDEF || heap == UNDEF) { *why = "the root group has no symbol table"; return false; }
        // local heap
        if (!in(heap, 32) || memcmp(d_.data() + base_ + heap, "HEAP", 4) != 0) { *why = "bad local heap"; return false; }
        const uint64_t hsize = raw(heap + 8, 8), hdata = raw(heap + 24, 8);
        if (!in(hdata, hsize)) { *why = "local heap data beyond the end of the file"; return false; }
        return walk(btree, hdata, hsize, 0, why);
    }

    bool walk(uint64_t node, uint64_t hdata, uint64_t hsize, int depth, std::string* why) {
        if (depth > 16 || !in(node, 24)) { *why = "bad group B-tree"; return false; }
        const uint8_t* q = d_.data() + base_ + node;
        if (memcmp(q, "TREE", 4) == 0) {
            if (q[4] != 0) { *why = "B-tree node is not a group node"; return false; }
            const int level = q[5];
            const unsigned used = (unsigned)raw(node + 6, 2);
            uint64_t a = node + 24 + 8;   // past key 0
            for (unsigned c = 0; c < used; c++, a += 16) {
                if (!in(a, 16)) { *why = "truncated B-tree node"; return false; }
                const uint64_t child = raw(a, 8);
                if (level > 0) { if (!walk(child, hdata, hsize, depth + 1, why)) return false; }
                else if (!snod(child, hdata, hsize, why)) return false;
            }
            return true;
        }
        *why = "bad group B-tree signature";
        return false;
    }

    bool snod(uint64_t node, uint64_t hdata, uint64_t hsize, std::string* why) {
        if (!in(node, 8) || memcmp(d_.data() + base_ + node, "SNOD", 4) != 0) { *why = "bad symbol table node"; return false; }
        const unsigned n = (unsigned)raw(node + 6, 2);
        for (unsigned i = 0; i < n; i++) {
            const uint64_t e = node + 8 + (uint64_t)i * ENTRY;
            if (!in(e, ENTRY)) { *why = "truncated symbol table node"; return false; }
            const uint64_t off = raw(e, 8), oh = raw(e + 8, 8);
            if (off >= hsize) { *why = "name offset past the local heap"; return false; }
            const char* s = (const char*)d_.data() + base_ + hdata + off;
            const size_t len = strnlen(s, hsize - off);
            ent_.emplace_back(std::string(s, len), oh);
        }
        return true;
    }

    // Parses the messages of a version-1 object header (following continuations).
    bool object(uint64_t oh, Info* info, std::string* why) {
        if (!in(oh, 16)) { *why = "object header beyond the end of the file"; return false; }
        if (d_[base_ + oh] != 1) { *why = "object header version " + std::to_string(d_[base_ + oh]) + " is not supported"; return false; }
        const unsigned nmsg = (unsigned)raw(oh + 2, 2);
        std::vector<std::pair<uint64_t, uint64_t>> chunks{{oh + 16, raw(oh + 8, 4)}};
        unsigned seen = 0;
        for (size_t c = 0; c < chunks.size() && c < 64; c++) {
            uint64_t a = chunks[c].first;
            const uint64_t end = a + chunks[c].second;
            if (!in(a, chunks[c].second)) { *why = "object header chunk beyond the end of the file"; return false; }
            while (a + 8 <= end && seen < nmsg) {
                const unsigned type = (unsigned)raw(a, 2), size = (unsigned)raw(a + 2, 2);
                const uint64_t m = a + 8;
                if (m + size > end) { *why = "object header message overruns its chunk"; return false; }
                seen++;
                if (type == 0x0001) {        // dataspace
                    const int v = d_[base_ + m], rank = d_[base_ + m + 1];
                    const uint64_t dims = m + (v == 1 ? 8 : 4);
                    size_t n = 1;
                    for (int r = 0; r < rank; r++) n *= (size_t)raw(dims + 8 * r, 8);
                    if (v == 2 && d_[base_ + m + 3] == 2) n = 0;   // null dataspace
                    info->nelem = n;
                    info->have_space = true;
                } else if (type == 0x0003) { // datatype
                    const int cls = d_[base_ + m] & 0x0f;
                    const uint8_t bits = d_[base_ + m + 1];
                    info->cls = cls;
                    info->esize = (size_t)raw(m + 4, 4);
                    info->big_endian = bits & 1;
                    info->is_signed = cls == 0 && (bits & 0x08);
                    if ((cls != 0 && cls != 1) || (cls == 1 && info->esize != 4 && info->esize != 8) ||
                        (cls == 0 && (info->esize < 1 || info->esize > 8))) {
                        *why = "datatype class " + std::to_string(cls) + " of size " + std::to_string(info->esize) + " is not supported";
                        return false;
                    }
                    info->have_type = true;
                } else if (type == 0x0008) { // data layout
                    const int v = d_[base_ + m];
                    if (v != 3 && v != 4) { *why = "data layout version " + std::to_string(v) + " is not supported"; return false; }
                    const int cls = d_[base_ + m + 1];
                    if (cls == 0) {          // compact
                        const unsigned cs = (unsigned)raw(m + 2, 2);
                        info->compact = true;
                        info->compact_data.assign(d_.begin() + base_ + m + 4, d_.begin() + base_ + m + 4 + cs);
                    } else if (cls == 1) {   // contiguous
                        info->addr = get(m + 2, 8);
                    } else { *why = "chunked or virtual storage is not supported"; return false; }
                    info->have_layout = true;
                } else if (type == 0x0011) { // symbol table
                    info->stab_btree = raw(m, 8);
                    info->stab_heap = raw(m + 8, 8);
                } else if (type == 0x0010) { // continuation
                    chunks.emplace_back(raw(m, 8), raw(m + 8, 8));
                }
                a = m + size;
            }
        }
        return true;
    }
};

}  // namespace spkh5
