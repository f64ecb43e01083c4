// HDF5 writer and reader for snapshot files; see h5lite.h. Structures and field orders follow the
// public HDF5 File Format Specification (superblock, object headers, header messages, version-1
// B-trees, symbol table nodes, local heaps); the code is this project's own.
#include "h5lite.h"

#include <algorithm>
#include <cstring>

namespace h5lite {

namespace {

constexpr uint64_t kUndef = ~0ull;
constexpr int kLeafK = 4, kInternalK = 16;            // group leaf / internal node K
constexpr uint16_t MSG_NIL = 0x0000, MSG_DATASPACE = 0x0001, MSG_LINKINFO = 0x0002, MSG_DATATYPE = 0x0003,
                   MSG_FILL = 0x0005, MSG_LINK = 0x0006, MSG_LAYOUT = 0x0008, MSG_ATTR = 0x000C,
                   MSG_CONT = 0x0010, MSG_SYMTAB = 0x0011, MSG_ATTRINFO = 0x0015;

size_t pad8(size_t n) { return (n + 7) & ~size_t(7); }

struct Buf {
    std::vector<uint8_t> b;
    size_t size() const { return b.size(); }
    void u8(uint8_t v) { b.push_back(v); }
    void le(uint64_t v, int n) { for (int k = 0; k < n; ++k) b.push_back((uint8_t)(v >> (8 * k))); }
    void bytes(const void* p, size_t n) { const uint8_t* q = (const uint8_t*)p; b.insert(b.end(), q, q + n); }
    void zeros(size_t n) { b.insert(b.end(), n, 0); }
    void align8() { zeros(pad8(b.size()) - b.size()); }
    void put_le(size_t at, uint64_t v, int n) { for (int k = 0; k < n; ++k) b[at + k] = (uint8_t)(v >> (8 * k)); }
};

// datatype message bodies (version 1): IEEE 754 binary64 little-endian, 32-bit signed integer
void type_f64(Buf& o) {
    o.u8(0x11);                          // version 1, class 1 (floating point)
    o.u8(0x20); o.u8(63); o.u8(0);       // little-endian, implied mantissa msb; sign at bit 63
    o.le(8, 4);                          // size
    o.le(0, 2); o.le(64, 2);             // bit offset, precision
    o.u8(52); o.u8(11); o.u8(0); o.u8(52);   // exponent location, size; mantissa location, size
    o.le(1023, 4);                       // exponent bias
}
void type_i32(Buf& o) {
    o.u8(0x10);                          // version 1, class 0 (fixed point)
    o.u8(0x08); o.u8(0); o.u8(0);        // little-endian, signed
    o.le(4, 4);
    o.le(0, 2); o.le(32, 2);             // bit offset, precision
}
constexpr size_t kTypeF64 = 20, kTypeI32 = 12;

// one header message of a version-1 object header: type, size, flags, 3 reserved bytes, body
void message(Buf& o, uint16_t type, const Buf& body, uint8_t flags = 0) {
    o.le(type, 2);
    o.le(pad8(body.size()), 2);
    o.u8(flags);
    o.zeros(3);
    o.bytes(body.b.data(), body.size());
    o.align8();
}

Buf attribute_body(const WriteAttr& a) {
    Buf o;
    o.u8(1); o.u8(0);                                    // version 1, reserved
    o.le(a.name.size() + 1, 2);
    o.le(a.is_int ? kTypeI32 : kTypeF64, 2);
    o.le(8, 2);                                          // dataspace message size (scalar)
    o.bytes(a.name.c_str(), a.name.size() + 1);
    o.align8();
    if (a.is_int) type_i32(o); else type_f64(o);
    o.align8();
    o.u8(1); o.u8(0); o.u8(0); o.zeros(5);               // dataspace version 1, rank 0: scalar
    if (a.is_int) o.le((uint32_t)a.i, 4);
    else { uint64_t u; std::memcpy(&u, &a.d, 8); o.le(u, 8); }
    return o;
}

// object header prefix (version 1): version, reserved, message count, reference count, size, pad
void header_prefix(Buf& o, int nmsg, size_t chunk) {
    o.u8(1); o.u8(0);
    o.le(nmsg, 2);
    o.le(1, 4);
    o.le(chunk, 4);
    o.zeros(4);
}

}  // namespace

bool write_file(const std::string& path, const std::vector<WriteDataset>& datasets,
                const std::vector<WriteAttr>& root_attrs, std::string& err) {
    if (datasets.size() > 2 * kLeafK) { err = "h5lite: at most 8 datasets per file"; return false; }
    std::vector<const WriteDataset*> ds;
    for (const auto& d : datasets) {
        if (d.name.empty() || d.name.size() > 255 || d.name.find('/') != std::string::npos) {
            err = "h5lite: bad dataset name '" + d.name + "'";
            return false;
        }
        ds.push_back(&d);
    }
    // symbol table entries are kept in name order (strcmp), as the B-tree keys require
    std::sort(ds.begin(), ds.end(), [](const WriteDataset* a, const WriteDataset* b) { return a->name < b->name; });
    for (size_t k = 1; k < ds.size(); ++k)
        if (ds[k]->name == ds[k - 1]->name) { err = "h5lite: duplicate dataset " + ds[k]->name; return false; }

    // ---- sizes, then addresses ----
    Buf root_msgs;                        // messages of the root group's object header
    {
        Buf sym;                          // B-tree and heap addresses, patched below
        sym.le(0, 8); sym.le(0, 8);
        message(root_msgs, MSG_SYMTAB, sym);
        for (const auto& a : root_attrs) message(root_msgs, MSG_ATTR, attribute_body(a));
    }
    const int root_nmsg = 1 + (int)root_attrs.size();
    std::vector<uint64_t> name_off;
    uint64_t heap_data_size = 8;          // offset 0: the empty name
    for (const auto* d : ds) { name_off.push_back(heap_data_size); heap_data_size += pad8(d->name.size() + 1); }
    const uint64_t btree_size = 24 + (2 * kInternalK + 1) * 8 + 2 * kInternalK * 8;
    const uint64_t snod_size = 8 + 2 * kLeafK * 40;
    std::vector<size_t> oh_chunk;
    for (const auto* d : ds) oh_chunk.push_back((8 + 8 + 8 * d->dims.size()) + (8 + pad8(kTypeF64)) + (8 + 8) + (8 + 24));

    const uint64_t a_root = 96;
    const uint64_t a_heap = a_root + 16 + root_msgs.size();
    const uint64_t a_heap_data = a_heap + 32;
    const uint64_t a_btree = a_heap_data + heap_data_size;
    const uint64_t a_snod = a_btree + btree_size;
    std::vector<uint64_t> a_oh(ds.size()), a_data(ds.size()), n_data(ds.size());
    uint64_t at = a_snod + snod_size;
    for (size_t k = 0; k < ds.size(); ++k) { a_oh[k] = at; at += 16 + oh_chunk[k]; }
    for (size_t k = 0; k < ds.size(); ++k) {
        uint64_t n = 1;
        for (uint64_t v : ds[k]->dims) n *= v;
        n_data[k] = n;
        a_data[k] = at;
        at += 8 * n;
    }
    const uint64_t eof = at;

    // ---- metadata ----
    Buf o;
    const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    o.bytes(sig, 8);
    o.u8(0); o.u8(0); o.u8(0); o.u8(0);          // superblock, free-space, root entry versions; reserved
    o.u8(0); o.u8(8); o.u8(8); o.u8(0);          // shared header version; sizes of offsets, lengths
    o.le(kLeafK, 2); o.le(kInternalK, 2);
    o.le(0, 4);                                  // file consistency flags
    o.le(0, 8); o.le(kUndef, 8); o.le(eof, 8); o.le(kUndef, 8);   // base, free space, end of file, driver
    o.le(0, 8); o.le(a_root, 8);                 // root symbol table entry: name offset, object header
    o.le(1, 4); o.le(0, 4);                      // cache type 1: B-tree and heap in the scratch pad
    o.le(a_btree, 8); o.le(a_heap, 8);
    // root group object header
    header_prefix(o, root_nmsg, root_msgs.size());
    const size_t sym_at = o.size() + 8;
    o.bytes(root_msgs.b.data(), root_msgs.size());
    o.put_le(sym_at, a_btree, 8);
    o.put_le(sym_at + 8, a_heap, 8);
    // local heap with the link names
    o.bytes("HEAP", 4); o.u8(0); o.zeros(3);
    o.le(heap_data_size, 8);
    o.le(1, 8);                                  // free-list head: none (1 marks the end of the list)
    o.le(a_heap_data, 8);
    o.zeros(8);
    for (const auto* d : ds) { o.bytes(d->name.c_str(), d->name.size() + 1); o.align8(); }
    // version-1 B-tree node of the group: one child (the symbol table node), keys = name offsets
    const size_t bt0 = o.size();
    o.bytes("TREE", 4); o.u8(0); o.u8(0);        // type 0 (group nodes), level 0
    o.le(ds.empty() ? 0 : 1, 2);
    o.le(kUndef, 8); o.le(kUndef, 8);            // no siblings
    if (!ds.empty()) { o.le(0, 8); o.le(a_snod, 8); o.le(name_off.back(), 8); }
    o.zeros(bt0 + btree_size - o.size());
    // symbol table node
    const size_t sn0 = o.size();
    o.bytes("SNOD", 4); o.u8(1); o.u8(0);
    o.le(ds.size(), 2);
    for (size_t k = 0; k < ds.size(); ++k) {
        o.le(name_off[k], 8); o.le(a_oh[k], 8);
        o.le(0, 4); o.le(0, 4); o.zeros(16);     // cache type 0: nothing cached
    }
    o.zeros(sn0 + snod_size - o.size());
    // dataset object headers
    for (size_t k = 0; k < ds.size(); ++k) {
        header_prefix(o, 4, oh_chunk[k]);
        Buf space;
        space.u8(1); space.u8((uint8_t)ds[k]->dims.size()); space.u8(0); space.zeros(5);
        for (uint64_t v : ds[k]->dims) space.le(v, 8);
        message(o, MSG_DATASPACE, space);
        Buf type;
        type_f64(type);
        message(o, MSG_DATATYPE, type, 1);       // constant
        Buf fill;
        fill.u8(2); fill.u8(2); fill.u8(2); fill.u8(0);   // version 2: late allocation, fill if set, none set
        message(o, MSG_FILL, fill, 1);
        Buf layout;
        layout.u8(3); layout.u8(1);              // version 3, contiguous
        layout.le(a_data[k], 8); layout.le(8 * n_data[k], 8);
        message(o, MSG_LAYOUT, layout);
    }
    if ((ds.empty() && o.size() != eof) || (!ds.empty() && o.size() != a_data[0])) {
        err = "h5lite: internal layout error";
        return false;
    }
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) { err = "cannot write " + path; return false; }
    bool ok = std::fwrite(o.b.data(), 1, o.size(), f) == o.size();
    for (size_t k = 0; ok && k < ds.size(); ++k) {
        // raw data: little-endian binary64, which is the host's layout on x86-64 and aarch64
        ok = std::fwrite(ds[k]->data, 8, n_data[k], f) == n_data[k];
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) err = "short write to " + path;
    return ok;
}

// ---------------------------------------------------------------------------------------------
// reader
// ---------------------------------------------------------------------------------------------
File::~File() {
    if (f_) std::fclose(f_);
}

bool File::read_at(uint64_t addr, void* dst, size_t n) const {
    if (addr == kUndef || addr + base_ + n > eof_) return false;
    if (fseeko(f_, (off_t)(addr + base_), SEEK_SET) != 0) return false;
    return std::fread(dst, 1, n, f_) == n;
}

uint64_t File::get_uint(const uint8_t* p, int n) const {
    uint64_t v = 0;
    for (int k = n - 1; k >= 0; --k) v = (v << 8) | p[k];
    if (n < 8 && v == (1ull << (8 * n)) - 1) return kUndef;   // all ones: the undefined address
    return v;
}

bool File::open(const std::string& path, std::string& err) {
    f_ = std::fopen(path.c_str(), "rb");
    if (!f_) { err = "cannot open " + path; return false; }
    fseeko(f_, 0, SEEK_END);
    const uint64_t fsize = (uint64_t)ftello(f_);
    eof_ = fsize;
    // the superblock sits at 0, 512, 1024, 2048, ... (after a user block)
    const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    uint64_t sb = kUndef;
    for (uint64_t a = 0; a + 8 <= fsize; a = a ? 2 * a : 512) {
        uint8_t s[8];
        base_ = 0;
        if (read_at(a, s, 8) && std::memcmp(s, sig, 8) == 0) { sb = a; break; }
    }
    if (sb == kUndef) { err = path + " is not an HDF5 file"; return false; }
    uint8_t h[128] = {0};
    const size_t hn = (size_t)std::min<uint64_t>(sizeof(h), fsize - sb);
    read_at(sb, h, hn);
    const int ver = h[8];
    uint64_t root_oh = kUndef, root_btree = kUndef, root_heap = kUndef;
    int cache = 0;
    if (ver == 0 || ver == 1) {
        so_ = h[13]; sl_ = h[14];
        if ((so_ != 4 && so_ != 8) || (sl_ != 4 && sl_ != 8)) { err = "unsupported offset size"; return false; }
        const uint8_t* p = h + 24 + (ver == 1 ? 4 : 0);
        base_ = get_uint(p, so_); p += so_;
        p += so_;                                       // free-space address
        const uint64_t e = get_uint(p, so_); p += so_;
        p += so_;                                       // driver information block
        p += so_;                                       // root entry: link name offset
        root_oh = get_uint(p, so_); p += so_;
        cache = (int)get_uint(p, 4); p += 8;
        if (cache == 1) { root_btree = get_uint(p, so_); root_heap = get_uint(p + so_, so_); }
        if (e != kUndef) eof_ = std::min<uint64_t>(fsize, e + base_);
    } else if (ver == 2 || ver == 3) {
        so_ = h[9]; sl_ = h[10];
        if ((so_ != 4 && so_ != 8) || (sl_ != 4 && sl_ != 8)) { err = "unsupported offset size"; return false; }
        const uint8_t* p = h + 12;
        base_ = get_uint(p, so_); p += so_;
        p += so_;                                       // superblock extension
        p += so_;                                       // end of file (not needed)
        root_oh = get_uint(p, so_);
    } else {
        err = "unsupported superblock version " + std::to_string(ver);
        return false;
    }
    std::vector<Msg> msgs;
    if (!object_header(root_oh, msgs, err)) return false;
    for (const Msg& m : msgs) {
        if (m.type == MSG_SYMTAB && m.data.size() >= (size_t)2 * so_) {
            root_btree = get_uint(m.data.data(), so_);
            root_heap = get_uint(m.data.data() + so_, so_);
        } else if (m.type == MSG_LINK) {
            const uint8_t* p = m.data.data();
            const uint8_t* end = p + m.data.size();
            if (p[0] != 1) { err = "unsupported link message version"; return false; }
            const uint8_t fl = p[1];
            p += 2;
            int ltype = 0;
            if (fl & 0x08) ltype = *p++;
            if (fl & 0x04) p += 8;
            if (fl & 0x10) p += 1;
            const int lsz = 1 << (fl & 3);
            const uint64_t nlen = get_uint(p, lsz);
            p += lsz;
            if (p + nlen > end) { err = "bad link message"; return false; }
            std::string name((const char*)p, (size_t)nlen);
            p += nlen;
            if (ltype == 0 && p + so_ <= end) links_[name] = get_uint(p, so_);
        } else if (m.type == MSG_LINKINFO) {
            // a fractal-heap address other than undefined means dense link storage
            const uint8_t* p = m.data.data();
            const uint8_t fl = p[1];
            p += 2 + ((fl & 1) ? 8 : 0);
            if (get_uint(p, so_) != kUndef) { err = "dense link storage is not supported"; return false; }
        } else if (m.type == MSG_ATTRINFO) {
            const uint8_t* p = m.data.data();
            const uint8_t fl = p[1];
            p += 2 + ((fl & 1) ? 2 : 0);
            if (get_uint(p, so_) != kUndef) { err = "dense attribute storage is not supported"; return false; }
        } else if (m.type == MSG_ATTR) {
            const uint8_t* p = m.data.data();
            const size_t n = m.data.size();
            if (n < 8) continue;
            const int av = p[0];
            if (av < 1 || av > 3) continue;
            if (av >= 2 && (p[1] & 3)) continue;                     // shared type or space
            const size_t name_len = p[2] | (p[3] << 8), dt_len = p[4] | (p[5] << 8), ds_len = p[6] | (p[7] << 8);
            size_t q = 8 + (av == 3 ? 1 : 0);
            const std::string name((const char*)p + q, strnlen((const char*)p + q, name_len));
            q += (av == 1) ? pad8(name_len) : name_len;
            Type t;
            if (q + dt_len > n || !decode_type(p + q, dt_len, t)) continue;
            q += (av == 1) ? pad8(dt_len) : dt_len;
            if (q + ds_len > n) continue;
            const uint8_t* s = p + q;
            const int rank = s[1];
            uint64_t count = 1;
            const int dv = s[0];
            const uint8_t* dims = s + (dv == 1 ? 8 : 4);
            if (dv == 2 && s[3] == 2) count = 0;                     // null dataspace
            for (int k = 0; k < rank; ++k) count *= get_uint(dims + k * sl_, sl_);
            q += (av == 1) ? pad8(ds_len) : ds_len;
            if (count != 1 || q + (size_t)t.size > n) continue;
            double v;
            if (convert(p + q, t, 1, &v)) attrs_[name] = v;
        }
    }
    if (root_btree != kUndef && root_heap != kUndef && !read_symbol_table(root_btree, root_heap, err)) return false;
    return true;
}

// object header of either version, continuation blocks followed; NIL messages dropped
bool File::object_header(uint64_t addr, std::vector<Msg>& out, std::string& err) const {
    uint8_t pre[16];
    if (!read_at(addr, pre, 16)) { err = "object header beyond the end of the file"; return false; }
    struct Chunk { uint64_t addr, len; bool v2, first; };
    std::vector<Chunk> todo;
    bool v2 = false, crt = false;
    if (std::memcmp(pre, "OHDR", 4) == 0) {
        v2 = true;
        if (pre[4] != 2) { err = "unsupported object header version"; return false; }
        const uint8_t fl = pre[5];
        crt = (fl & 0x04) != 0;
        uint64_t p = 6 + ((fl & 0x20) ? 16 : 0) + ((fl & 0x10) ? 4 : 0);
        uint8_t sz[8] = {0};
        const int nb = 1 << (fl & 3);
        if (!read_at(addr + p, sz, nb)) { err = "bad object header"; return false; }
        uint64_t len = 0;
        for (int k = nb - 1; k >= 0; --k) len = (len << 8) | sz[k];
        todo.push_back({addr + p + nb, len, true, true});
    } else {
        if (pre[0] != 1) { err = "unsupported object header version " + std::to_string(pre[0]); return false; }
        const uint64_t len = pre[8] | (pre[9] << 8) | (pre[10] << 16) | ((uint64_t)pre[11] << 24);
        todo.push_back({addr + 16, len, false, true});
    }
    for (size_t c = 0; c < todo.size() && c < 1000; ++c) {
        Chunk ch = todo[c];
        std::vector<uint8_t> b(ch.len);
        if (!read_at(ch.addr, b.data(), ch.len)) { err = "object header chunk beyond the end of the file"; return false; }
        size_t p = 0, end = ch.len;
        if (v2) {
            if (!ch.first) {
                if (ch.len < 8 || std::memcmp(b.data(), "OCHK", 4) != 0) { err = "bad continuation chunk"; return false; }
                p = 4;
            }
            // chunk 0's length counts its messages only (its checksum follows); a continuation
            // block's counts the signature and the 4-byte checksum at its end
            if (!ch.first) end = ch.len - 4;
        }
        const size_t hdr = v2 ? (4 + (crt ? 2 : 0)) : 8;
        while (p + hdr <= end) {
            Msg m;
            size_t n;
            if (v2) {
                m.type = b[p];
                n = b[p + 1] | (b[p + 2] << 8);
                m.flags = b[p + 3];
            } else {
                m.type = b[p] | (b[p + 1] << 8);
                n = b[p + 2] | (b[p + 3] << 8);
                m.flags = b[p + 4];
            }
            p += hdr;
            if (p + n > end) { err = "object header message overruns its chunk"; return false; }
            m.data.assign(b.begin() + p, b.begin() + p + n);
            p += n;
            if (m.type == MSG_CONT) {
                if (n < (size_t)(so_ + sl_)) { err = "bad continuation message"; return false; }
                todo.push_back({get_uint(m.data.data(), so_), get_uint(m.data.data() + so_, sl_), v2, false});
            } else if (m.type != MSG_NIL) {
                if (m.flags & 0x02) {
                    if (m.type == MSG_DATATYPE || m.type == MSG_DATASPACE) { err = "shared messages are not supported"; return false; }
                }
                out.push_back(std::move(m));
            }
        }
    }
    return true;
}

bool File::read_symbol_table(uint64_t btree, uint64_t heap, std::string& err) {
    uint8_t h[40];
    if (!read_at(heap, h, 8 + 2 * sl_ + so_) || std::memcmp(h, "HEAP", 4) != 0) { err = "bad local heap"; return false; }
    const uint64_t data = get_uint(h + 8 + 2 * sl_, so_);
    return btree_node(btree, data, 0, err);
}

bool File::btree_node(uint64_t addr, uint64_t heap_data, int depth, std::string& err) {
    if (depth > 32) { err = "B-tree too deep"; return false; }
    uint8_t h[8];
    if (!read_at(addr, h, 8)) { err = "B-tree node beyond the end of the file"; return false; }
    if (std::memcmp(h, "TREE", 4) == 0) {
        if (h[4] != 0) { err = "not a group B-tree"; return false; }
        const int level = h[5];
        const int n = h[6] | (h[7] << 8);
        const size_t len = 2 * so_ + (size_t)(2 * n + 1) * sl_ + (size_t)n * so_;
        std::vector<uint8_t> b(len);
        if (!read_at(addr + 8, b.data(), len)) { err = "truncated B-tree node"; return false; }
        size_t p = 2 * so_ + sl_;                             // siblings, key 0
        for (int k = 0; k < n; ++k) {
            const uint64_t child = get_uint(b.data() + p, so_);
            p += so_ + sl_;
            (void)level;                                      // children: B-tree nodes, or symbol table nodes at level 0
            if (!btree_node(child, heap_data, depth + 1, err)) return false;
        }
        return true;
    }
    if (std::memcmp(h, "SNOD", 4) == 0) {
        const int n = h[6] | (h[7] << 8);
        const size_t ent = 2 * so_ + 8 + 16;
        std::vector<uint8_t> b((size_t)n * ent);
        if (!read_at(addr + 8, b.data(), b.size())) { err = "truncated symbol table node"; return false; }
        for (int k = 0; k < n; ++k) {
            const uint8_t* e = b.data() + (size_t)k * ent;
            const uint64_t off = get_uint(e, so_), oh = get_uint(e + so_, so_);
            char name[256] = {0};
            uint64_t len = std::min<uint64_t>(255, eof_ - base_ - (heap_data + off));
            read_at(heap_data + off, name, (size_t)len);
            links_[std::string(name, strnlen(name, 255))] = oh;
        }
        return true;
    }
    err = "bad group node";
    return false;
}

bool File::decode_type(const uint8_t* p, size_t n, Type& t) const {
    if (n < 8) return false;
    t.cls = p[0] & 0x0f;
    t.size = (int)(p[4] | (p[5] << 8) | (p[6] << 16) | ((uint32_t)p[7] << 24));
    if (t.cls == 0) {
        t.big_endian = p[1] & 1;
        t.is_signed = (p[1] >> 3) & 1;
        return t.size == 1 || t.size == 2 || t.size == 4 || t.size == 8;
    }
    if (t.cls == 1) {
        if (p[1] & 0x40) return false;                    // VAX order
        t.big_endian = p[1] & 1;
        return t.size == 4 || t.size == 8;
    }
    return false;
}

bool File::convert(const uint8_t* src, const Type& t, uint64_t count, double* dst) const {
    const int s = t.size;
    for (uint64_t k = 0; k < count; ++k) {
        uint8_t b[8];
        for (int q = 0; q < s; ++q) b[q] = t.big_endian ? src[k * s + (s - 1 - q)] : src[k * s + q];
        if (t.cls == 1) {
            if (s == 8) { double v; std::memcpy(&v, b, 8); dst[k] = v; }
            else { float v; std::memcpy(&v, b, 4); dst[k] = v; }
        } else {
            uint64_t u = 0;
            for (int q = s - 1; q >= 0; --q) u = (u << 8) | b[q];
            if (t.is_signed && s < 8 && (u >> (8 * s - 1)) & 1) u |= ~0ull << (8 * s);
            dst[k] = t.is_signed ? (double)(int64_t)u : (double)u;
        }
    }
    return true;
}

bool File::attr(const std::string& name, double& v) const {
    auto it = attrs_.find(name);
    if (it == attrs_.end()) return false;
    v = it->second;
    return true;
}

bool File::read(const std::string& name, std::vector<uint64_t>& dims, std::vector<double>& out, std::string& err) {
    auto it = links_.find(name);
    if (it == links_.end()) { err = "no dataset " + name; return false; }
    std::vector<Msg> msgs;
    if (!object_header(it->second, msgs, err)) return false;
    Type t;
    bool have_t = false, have_s = false, have_l = false;
    uint64_t daddr = kUndef, dsize = 0;
    std::vector<uint8_t> compact;
    dims.clear();
    for (const Msg& m : msgs) {
        const uint8_t* p = m.data.data();
        if (m.type == MSG_DATATYPE) {
            if (!decode_type(p, m.data.size(), t)) { err = name + ": unsupported datatype"; return false; }
            have_t = true;
        } else if (m.type == MSG_DATASPACE) {
            const int v = p[0], rank = p[1];
            const uint8_t* d = p + (v == 1 ? 8 : 4);
            if (v == 2 && p[3] == 2) { err = name + ": null dataspace"; return false; }
            for (int k = 0; k < rank; ++k) dims.push_back(get_uint(d + k * sl_, sl_));
            have_s = true;
        } else if (m.type == MSG_LAYOUT) {
            const int v = p[0];
            if (v != 3 && v != 4) { err = name + ": unsupported layout message version"; return false; }
            const int cls = p[1];
            if (cls == 1) { daddr = get_uint(p + 2, so_); dsize = get_uint(p + 2 + so_, sl_); }
            else if (cls == 0) {
                const size_t n = p[2] | (p[3] << 8);
                compact.assign(p + 4, p + 4 + n);
            } else { err = name + ": chunked or virtual storage is not supported"; return false; }
            have_l = true;
        } else if (m.type == 0x000B) {
            err = name + ": filtered (compressed) data is not supported";
            return false;
        }
    }
    if (!have_t || !have_s || !have_l) { err = name + ": not a dataset"; return false; }
    uint64_t count = 1;
    for (uint64_t d : dims) count *= d;
    const uint64_t bytes = count * (uint64_t)t.size;
    std::vector<uint8_t> raw(bytes, 0);
    if (!compact.empty()) {
        if (compact.size() < bytes) { err = name + ": short compact data"; return false; }
        std::memcpy(raw.data(), compact.data(), bytes);
    } else if (daddr != kUndef) {
        if (dsize < bytes || !read_at(daddr, raw.data(), bytes)) { err = name + ": data beyond the end of the file"; return false; }
    }
    out.resize(count);
    return convert(raw.data(), t, count, out.data());
}

}  // namespace h5lite
