// h5lite: see h5lite.hpp.  Layout written (all addresses 8 bytes, all lengths 8 bytes):
//   superblock v0 with the root group's symbol-table entry (cache type 1: B-tree and heap address)
//   for every group: its datasets (raw data, then a v1 object header each), its subgroups, a local
//     heap with the names, symbol-table nodes of up to 8 entries sorted by name, one level-0 B-tree
//     node over them (up to 32), and the group's v1 object header with a symbol-table message
//   dataset object header: dataspace (v1), datatype (v1: 32-bit signed LE integer or IEEE double
//     LE), fill value (v2, none defined), data layout (v3, contiguous).
#include "h5lite.hpp"

#include <algorithm>
#include <cstring>
#include <fstream>
#include <functional>
#include <sstream>

namespace h5lite {
namespace {

constexpr uint64_t UNDEF = ~0ull;
constexpr int LEAF_K = 4;       // symbol-table node: up to 2 * 4 entries
constexpr int INTERNAL_K = 16;  // B-tree node: up to 2 * 16 children
const uint8_t SIG[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};

size_t esize(Type t) { return t == Type::I32 ? 4 : 8; }

struct Buf {
    std::vector<uint8_t> b;
    size_t tell() const { return b.size(); }
    void align8() {
        while (b.size() % 8) b.push_back(0);
    }
    void u8(uint64_t v) { b.push_back((uint8_t)v); }
    void u16(uint64_t v) { put(v, 2); }
    void u32(uint64_t v) { put(v, 4); }
    void u64(uint64_t v) { put(v, 8); }
    void put(uint64_t v, int n) {
        for (int i = 0; i < n; ++i) b.push_back((uint8_t)(v >> (8 * i)));
    }
    void bytes(const void* p, size_t n) {
        const uint8_t* q = static_cast<const uint8_t*>(p);
        b.insert(b.end(), q, q + n);
    }
    void zeros(size_t n) { b.insert(b.end(), n, 0); }
    void patch64(size_t at, uint64_t v) {
        for (int i = 0; i < 8; ++i) b[at + i] = (uint8_t)(v >> (8 * i));
    }
};

struct Msg {
    uint16_t type;
    std::vector<uint8_t> data;
};

// v1 object header with the given messages; returns its address.
uint64_t put_ohdr(Buf& f, const std::vector<Msg>& msgs) {
    f.align8();
    const uint64_t at = f.tell();
    size_t body = 0;
    for (const auto& m : msgs) body += 8 + ((m.data.size() + 7) / 8) * 8;
    f.u8(1);
    f.u8(0);
    f.u16(msgs.size());
    f.u32(1);  // reference count
    f.u32(body);
    f.u32(0);  // alignment of the messages to 8 bytes
    for (const auto& m : msgs) {
        const size_t sz = ((m.data.size() + 7) / 8) * 8;
        f.u16(m.type);
        f.u16(sz);
        f.u8(0);
        f.zeros(3);
        f.bytes(m.data.data(), m.data.size());
        f.zeros(sz - m.data.size());
    }
    return at;
}

std::vector<uint8_t> le(std::initializer_list<std::pair<uint64_t, int>> fields) {
    Buf b;
    for (const auto& fl : fields) b.put(fl.first, fl.second);
    return b.b;
}

uint64_t put_dataset(Buf& f, const Dataset& d) {
    f.align8();
    const uint64_t daddr = f.tell();
    f.bytes(d.data.data(), d.data.size());
    std::vector<Msg> m;
    {  // dataspace v1
        Buf b;
        b.u8(1);
        b.u8(d.dims.size());
        b.u8(0);
        b.u8(0);
        b.u32(0);
        for (auto x : d.dims) b.u64(x);
        m.push_back({0x0001, b.b});
    }
    if (d.type == Type::I32) {  // fixed point, signed, little endian
        m.push_back({0x0003, le({{0x10, 1}, {0x08, 1}, {0, 2}, {4, 4}, {0, 2}, {32, 2}})});
    } else {  // IEEE double, little endian
        m.push_back({0x0003, le({{0x11, 1}, {0x20, 1}, {63, 1}, {0, 1}, {8, 4}, {0, 2}, {64, 2}, {52, 1}, {11, 1},
                                 {0, 1}, {52, 1}, {1023, 4}})});
    }
    m.push_back({0x0005, le({{2, 1}, {2, 1}, {2, 1}, {0, 1}})});  // fill value v2: late, if set, none
    m.push_back({0x0008, le({{3, 1}, {1, 1}, {daddr, 8}, {d.data.size(), 8}})});  // contiguous layout v3
    return put_ohdr(f, m);
}

struct GroupAddr {
    uint64_t ohdr, btree, heap;
};

GroupAddr put_group(Buf& f, const Group& g) {
    struct Ent {
        std::string name;
        uint64_t ohdr;
        bool group;
        uint64_t btree, heap;
    };
    std::vector<Ent> ents;
    for (const auto& kv : g.datasets) ents.push_back({kv.first, put_dataset(f, kv.second), false, 0, 0});
    for (const auto& kv : g.groups) {
        const GroupAddr a = put_group(f, *kv.second);
        ents.push_back({kv.first, a.ohdr, true, a.btree, a.heap});
    }
    std::sort(ents.begin(), ents.end(), [](const Ent& a, const Ent& b) { return a.name < b.name; });
    if (ents.size() > (size_t)2 * LEAF_K * 2 * INTERNAL_K) throw std::runtime_error("h5lite: too many members in a group");
    // local heap: the empty name at offset 0, then every name, 8-byte padded
    std::vector<uint8_t> heapdata(8, 0);
    std::vector<uint64_t> noff;
    for (const auto& e : ents) {
        noff.push_back(heapdata.size());
        heapdata.insert(heapdata.end(), e.name.begin(), e.name.end());
        heapdata.push_back(0);
        while (heapdata.size() % 8) heapdata.push_back(0);
    }
    f.align8();
    const uint64_t heapdata_addr = f.tell();
    f.bytes(heapdata.data(), heapdata.size());
    f.align8();
    const uint64_t heap = f.tell();
    f.bytes("HEAP", 4);
    f.u8(0);
    f.zeros(3);
    f.u64(heapdata.size());
    f.u64(UNDEF);  // no free block
    f.u64(heapdata_addr);
    // symbol-table nodes
    std::vector<uint64_t> snods, lastkey;
    for (size_t i0 = 0; i0 < ents.size() || (i0 == 0 && ents.empty()); i0 += 2 * LEAF_K) {
        const size_t i1 = std::min(ents.size(), i0 + 2 * LEAF_K);
        f.align8();
        snods.push_back(f.tell());
        f.bytes("SNOD", 4);
        f.u8(1);
        f.u8(0);
        f.u16(i1 - i0);
        for (size_t i = i0; i < i0 + 2 * LEAF_K; ++i) {
            if (i < i1) {
                const Ent& e = ents[i];
                f.u64(noff[i]);
                f.u64(e.ohdr);
                f.u32(e.group ? 1 : 0);
                f.u32(0);
                f.u64(e.group ? e.btree : 0);
                f.u64(e.group ? e.heap : 0);
            } else {
                f.zeros(40);
            }
        }
        lastkey.push_back(i1 > i0 ? noff[i1 - 1] : 0);
        if (ents.empty()) break;
    }
    // one level-0 B-tree node over the symbol-table nodes
    f.align8();
    const uint64_t btree = f.tell();
    f.bytes("TREE", 4);
    f.u8(0);  // group node
    f.u8(0);  // level
    f.u16(ents.empty() ? 0 : snods.size());
    f.u64(UNDEF);
    f.u64(UNDEF);
    for (int i = 0; i < 2 * INTERNAL_K; ++i) {
        f.u64(i == 0 ? 0 : (i - 1 < (int)lastkey.size() ? lastkey[i - 1] : 0));  // key i
        f.u64(i < (int)snods.size() && !ents.empty() ? snods[i] : 0);       // child i
    }
    f.u64(!lastkey.empty() ? lastkey.back() : 0);  // key 2K
    // the group's object header: one symbol-table message
    std::vector<Msg> m;
    m.push_back({0x0011, le({{btree, 8}, {heap, 8}})});
    const uint64_t oh = put_ohdr(f, m);
    return {oh, btree, heap};
}

// ------------------------------------------------------------------ reader
struct Reader {
    std::vector<uint8_t> b;
    std::string err;
    uint64_t base = 0;
    bool ok(uint64_t at, uint64_t n) const { return at <= b.size() && n <= b.size() - at; }
    uint64_t get(uint64_t at, int n) {
        if (!ok(at, n)) throw std::runtime_error("read past the end of the file");
        uint64_t v = 0;
        for (int i = 0; i < n; ++i) v |= (uint64_t)b[at + i] << (8 * i);
        return v;
    }
    std::string cstr(uint64_t at) {
        std::string s;
        while (ok(at, 1) && b[at]) s.push_back((char)b[at++]);
        return s;
    }
};

struct ObjInfo {
    bool is_group = false;
    uint64_t btree = 0, heap = 0;
    bool has_space = false, has_type = false, has_layout = false;
    std::vector<uint64_t> dims;
    int tclass = -1;
    uint64_t tsize = 0;
    bool tsigned = true, big_endian = false;
    uint64_t data_addr = UNDEF, data_size = 0;
    std::vector<uint8_t> compact;
    bool is_compact = false;
};

void parse_messages(Reader& r, uint64_t at, uint64_t len, int nmsg_left, ObjInfo& o, int depth);

void parse_msg(Reader& r, uint16_t type, uint64_t d, uint64_t sz, ObjInfo& o, int depth) {
    switch (type) {
        case 0x0001: {  // dataspace
            const int ver = (int)r.get(d, 1), rank = (int)r.get(d + 1, 1);
            const uint64_t p = d + (ver == 1 ? 8 : 4);
            o.dims.clear();
            for (int i = 0; i < rank; ++i) o.dims.push_back(r.get(p + 8 * i, 8));
            o.has_space = true;
            break;
        }
        case 0x0003: {  // datatype
            const int cv = (int)r.get(d, 1);
            o.tclass = cv & 15;
            const uint64_t bits = r.get(d + 1, 3);
            o.tsize = r.get(d + 4, 4);
            o.big_endian = bits & 1;
            o.tsigned = o.tclass == 0 ? ((bits >> 3) & 1) : true;
            o.has_type = true;
            break;
        }
        case 0x0008: {  // data layout
            const int ver = (int)r.get(d, 1);
            if (ver != 3) throw std::runtime_error("data layout message version " + std::to_string(ver) + " not handled");
            const int cls = (int)r.get(d + 1, 1);
            if (cls == 1) {
                o.data_addr = r.get(d + 2, 8);
                o.data_size = r.get(d + 10, 8);
            } else if (cls == 0) {
                const uint64_t n = r.get(d + 2, 2);
                if (!r.ok(d + 4, n)) throw std::runtime_error("compact data past the end of the file");
                o.compact.assign(r.b.begin() + d + 4, r.b.begin() + d + 4 + n);
                o.is_compact = true;
                o.data_size = n;
            } else {
                throw std::runtime_error("chunked or virtual datasets are not handled");
            }
            o.has_layout = true;
            break;
        }
        case 0x0011:  // symbol table
            o.is_group = true;
            o.btree = r.get(d, 8);
            o.heap = r.get(d + 8, 8);
            break;
        case 0x0010: {  // continuation
            const uint64_t caddr = r.get(d, 8), clen = r.get(d + 8, 8);
            if (depth > 16) throw std::runtime_error("object header continuation chain too long");
            parse_messages(r, caddr, clen, 1 << 20, o, depth + 1);
            break;
        }
        case 0x000b:  // filter pipeline
            throw std::runtime_error("filtered (compressed) datasets are not handled");
        default:
            break;  // fill values, times, attributes, NULL: not needed
    }
    (void)sz;
}

void parse_messages(Reader& r, uint64_t at, uint64_t len, int nmsg_left, ObjInfo& o, int depth) {
    uint64_t p = at;
    while (p + 8 <= at + len && nmsg_left-- > 0) {
        const uint16_t type = (uint16_t)r.get(p, 2);
        const uint64_t sz = r.get(p + 2, 2);
        parse_msg(r, type, p + 8, sz, o, depth);
        p += 8 + sz;
    }
}

ObjInfo parse_object(Reader& r, uint64_t at) {
    ObjInfo o;
    if (r.ok(at, 4) && std::memcmp(&r.b[at], "OHDR", 4) == 0)
        throw std::runtime_error("version 2 object headers are not handled (file written with the latest format)");
    const int ver = (int)r.get(at, 1);
    if (ver != 1) throw std::runtime_error("object header version " + std::to_string(ver) + " not handled");
    const int nmsg = (int)r.get(at + 2, 2);
    const uint64_t size = r.get(at + 8, 4);
    parse_messages(r, at + 16, size, nmsg, o, 0);
    return o;
}

void read_group(Reader& r, uint64_t btree, uint64_t heap, Group& g, int depth);

void read_entry(Reader& r, uint64_t heapdata, uint64_t e, Group& g, int depth) {
    const std::string name = r.cstr(heapdata + r.get(e, 8));
    const uint64_t oh = r.get(e + 8, 8);
    ObjInfo o = parse_object(r, oh);
    if (o.is_group) {
        read_group(r, o.btree, o.heap, g.group(name), depth + 1);
        return;
    }
    if (!o.has_space || !o.has_type || !o.has_layout) return;  // not a dataset of this subset
    Dataset d;
    if (o.tclass == 0 && o.tsize == 4 && o.tsigned) d.type = Type::I32;
    else if (o.tclass == 1 && o.tsize == 8) d.type = Type::F64;
    else if (o.tclass == 0 && o.tsize == 8 && o.tsigned) d.type = Type::I32;  // 64-bit integers: narrowed below
    else throw std::runtime_error("dataset " + name + ": datatype not handled (32/64-bit integer or double)");
    if (o.big_endian) throw std::runtime_error("dataset " + name + ": big-endian data not handled");
    d.dims = o.dims;
    const size_t n = d.count();
    if (o.tclass == 0 && o.tsize == 8) {  // 64-bit integers -> 32-bit
        std::vector<int32_t> v(n);
        for (size_t i = 0; i < n; ++i) v[i] = (int32_t)(o.is_compact ? 0 : r.get(o.data_addr + 8 * i, 8));
        d.data.assign(reinterpret_cast<uint8_t*>(v.data()), reinterpret_cast<uint8_t*>(v.data()) + 4 * n);
    } else {
        const size_t bytes = n * esize(d.type);
        if (o.is_compact) {
            if (o.compact.size() < bytes) throw std::runtime_error("dataset " + name + ": short compact data");
            d.data.assign(o.compact.begin(), o.compact.begin() + bytes);
        } else if (o.data_addr == UNDEF) {
            d.data.assign(bytes, 0);  // never written: the (zero) fill value
        } else {
            if (!r.ok(o.data_addr, bytes)) throw std::runtime_error("dataset " + name + ": data past the end of the file");
            d.data.assign(r.b.begin() + o.data_addr, r.b.begin() + o.data_addr + bytes);
        }
    }
    g.datasets[name] = std::move(d);
}

void read_btree(Reader& r, uint64_t node, uint64_t heapdata, Group& g, int depth) {
    if (!r.ok(node, 24) || std::memcmp(&r.b[node], "TREE", 4) != 0) throw std::runtime_error("bad B-tree node");
    const int level = (int)r.get(node + 5, 1);
    const int used = (int)r.get(node + 6, 2);
    for (int i = 0; i < used; ++i) {
        const uint64_t child = r.get(node + 24 + 8 + 16 * i, 8);
        if (level > 0) {
            read_btree(r, child, heapdata, g, depth);
        } else {
            if (!r.ok(child, 8) || std::memcmp(&r.b[child], "SNOD", 4) != 0) throw std::runtime_error("bad symbol-table node");
            const int ns = (int)r.get(child + 6, 2);
            for (int k = 0; k < ns; ++k) read_entry(r, heapdata, child + 8 + 40 * k, g, depth);
        }
    }
}

void read_group(Reader& r, uint64_t btree, uint64_t heap, Group& g, int depth) {
    if (depth > 32) throw std::runtime_error("groups nested too deeply");
    if (!r.ok(heap, 32) || std::memcmp(&r.b[heap], "HEAP", 4) != 0) throw std::runtime_error("bad local heap");
    const uint64_t heapdata = r.get(heap + 24, 8);
    read_btree(r, btree, heapdata, g, depth);
}

}  // namespace

Dataset make_f64(const double* a, const std::vector<uint64_t>& fd) {
    Dataset d;
    d.type = Type::F64;
    d.dims.assign(fd.rbegin(), fd.rend());
    d.data.assign(reinterpret_cast<const uint8_t*>(a), reinterpret_cast<const uint8_t*>(a) + 8 * d.count());
    return d;
}
Dataset make_i32(const int32_t* a, const std::vector<uint64_t>& fd) {
    Dataset d;
    d.type = Type::I32;
    d.dims.assign(fd.rbegin(), fd.rend());
    d.data.assign(reinterpret_cast<const uint8_t*>(a), reinterpret_cast<const uint8_t*>(a) + 4 * d.count());
    return d;
}
std::vector<uint64_t> fortran_dims(const Dataset& d) { return std::vector<uint64_t>(d.dims.rbegin(), d.dims.rend()); }

std::string write_file(const std::string& path, const Group& root) {
    try {
        Buf f;
        // superblock v0 (patched at the end)
        f.bytes(SIG, 8);
        f.u8(0); f.u8(0); f.u8(0); f.u8(0);  // superblock, free space, root entry, reserved
        f.u8(0); f.u8(8); f.u8(8); f.u8(0);  // shared header version, offset and length sizes
        f.u16(LEAF_K);
        f.u16(INTERNAL_K);
        f.u32(0);                            // consistency flags
        f.u64(0);                            // base address
        f.u64(UNDEF);                        // free-space info
        const size_t eof_at = f.tell();
        f.u64(0);                            // end of file (patched)
        f.u64(UNDEF);                        // driver information
        const size_t root_at = f.tell();     // root symbol-table entry (patched)
        f.zeros(40);
        const GroupAddr r = put_group(f, root);
        f.align8();
        f.patch64(eof_at, f.tell());
        f.patch64(root_at, 0);
        f.patch64(root_at + 8, r.ohdr);
        f.b[root_at + 16] = 1;  // cache type 1: B-tree and heap in the scratch pad
        f.patch64(root_at + 24, r.btree);
        f.patch64(root_at + 32, r.heap);
        std::ofstream o(path, std::ios::binary | std::ios::trunc);
        if (!o) return "cannot create " + path;
        o.write(reinterpret_cast<const char*>(f.b.data()), (std::streamsize)f.b.size());
        if (!o) return "write failed: " + path;
        return "";
    } catch (const std::exception& e) {
        return e.what();
    }
}

std::string read_file(const std::string& path, Group& root) {
    Reader r;
    {
        std::ifstream in(path, std::ios::binary);
        if (!in) return "cannot open " + path;
        r.b.assign(std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>());
    }
    try {
        // the superblock sits at 0, 512, 1024, ... (a user block may precede it)
        uint64_t sb = UNDEF;
        for (uint64_t at = 0; at + 8 <= r.b.size(); at = at ? 2 * at : 512)
            if (std::memcmp(&r.b[at], SIG, 8) == 0) {
                sb = at;
                break;
            }
        if (sb == UNDEF) return path + ": not an HDF5 file";
        const int ver = (int)r.get(sb + 8, 1);
        if (ver > 1) return path + ": superblock version " + std::to_string(ver) + " not handled";
        if (r.get(sb + 13, 1) != 8 || r.get(sb + 14, 1) != 8) return path + ": only 8-byte offsets and lengths are handled";
        uint64_t p = sb + 24 + (ver == 1 ? 4 : 0);  // after the K values (and v1's indexed-storage K)
        p += 8 * 4;                                  // base, free space, end of file, driver
        const uint64_t oh = r.get(p + 8, 8);
        ObjInfo o = parse_object(r, oh);
        if (!o.is_group) return path + ": root object is not a symbol-table group";
        read_group(r, o.btree, o.heap, root, 0);
        return "";
    } catch (const std::exception& e) {
        return path + ": " + e.what();
    }
}

}  // namespace h5lite
