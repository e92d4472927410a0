// HDF5 writer and reader for the reference's output layout (see h5file.h). Structures and field
// orders follow "HDF5 File Format Specification" (The HDF Group): superblock version 0, object
// header version 1, group B-tree (type 0) version 1 nodes, symbol-table nodes, local heaps, and
// the dataspace, datatype, fill-value, data-layout (version 3), modification-time, attribute,
// continuation and symbol-table messages.
#include "h5file.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iterator>

namespace thorx_h5 {
namespace {

constexpr uint64_t kUndef     = 0xFFFFFFFFFFFFFFFFull;
constexpr int      kLeafK     = 4;  // the library's default group leaf K
constexpr int      kInternalK = 16; // and internal-node K
constexpr int      kSnodCap   = 2 * kLeafK;
constexpr int      kBtreeCap  = 2 * kInternalK;
const uint8_t      kSignature[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};

enum : uint16_t {
    kMsgNil = 0x0, kMsgDataspace = 0x1, kMsgDatatype = 0x3, kMsgFill = 0x5, kMsgLayout = 0x8,
    kMsgAttribute = 0xC, kMsgContinuation = 0x10, kMsgSymtab = 0x11, kMsgMtime = 0x12
};

using Bytes = std::vector<uint8_t>;

template<class T>
void put(Bytes& b, T v) { // little-endian
    for (size_t i = 0; i < sizeof(T); i++)
        b.push_back((uint8_t)((uint64_t)v >> (8 * i)));
}
void put_bytes(Bytes& b, const void* p, size_t n) {
    const uint8_t* q = (const uint8_t*)p;
    b.insert(b.end(), q, q + n);
}
void pad8(Bytes& b) {
    while (b.size() % 8)
        b.push_back(0);
}
template<class T>
void poke(Bytes& b, size_t at, T v) {
    for (size_t i = 0; i < sizeof(T); i++)
        b[at + i] = (uint8_t)((uint64_t)v >> (8 * i));
}

// a message of an object header v1: type, size of the body padded to 8, flags, 3 reserved bytes
Bytes message(uint16_t type, Bytes body, uint8_t flags = 0) {
    pad8(body);
    Bytes m;
    put<uint16_t>(m, type);
    put<uint16_t>(m, (uint16_t)body.size());
    put<uint8_t>(m, flags);
    put<uint8_t>(m, 0), put<uint8_t>(m, 0), put<uint8_t>(m, 0);
    put_bytes(m, body.data(), body.size());
    return m;
}

// datatype messages (v1) of the two numeric types, and of a fixed-length null-terminated string
Bytes dt_f64() {
    Bytes b = {0x11, 0x20, 0x3F, 0x00};
    put<uint32_t>(b, 8);
    put<uint16_t>(b, 0), put<uint16_t>(b, 64);
    put<uint8_t>(b, 52), put<uint8_t>(b, 11), put<uint8_t>(b, 0), put<uint8_t>(b, 52);
    put<uint32_t>(b, 1023);
    return b;
}
Bytes dt_i32() {
    Bytes b = {0x10, 0x08, 0x00, 0x00};
    put<uint32_t>(b, 4);
    put<uint16_t>(b, 0), put<uint16_t>(b, 32);
    return b;
}
Bytes dt_string(uint32_t n) {
    Bytes b = {0x13, 0x00, 0x00, 0x00};
    put<uint32_t>(b, n);
    return b;
}
const Bytes kScalarSpace = {1, 0, 0, 0, 0, 0, 0, 0}; // dataspace v1, rank 0

// attribute message v1: a scalar fixed-length string (an empty text is one null byte)
Bytes attribute(const std::string& name, const std::string& text) {
    Bytes data(text.begin(), text.end());
    if (data.empty())
        data.push_back(0);
    Bytes nm(name.begin(), name.end());
    nm.push_back(0);
    const Bytes dt = dt_string((uint32_t)data.size());
    Bytes       b;
    put<uint8_t>(b, 1), put<uint8_t>(b, 0);
    put<uint16_t>(b, (uint16_t)nm.size());
    put<uint16_t>(b, (uint16_t)dt.size());
    put<uint16_t>(b, (uint16_t)kScalarSpace.size());
    put_bytes(b, nm.data(), nm.size()), pad8(b);
    put_bytes(b, dt.data(), dt.size()), pad8(b);
    put_bytes(b, kScalarSpace.data(), kScalarSpace.size()), pad8(b);
    put_bytes(b, data.data(), data.size());
    return message(kMsgAttribute, b);
}

// the dataset's messages in the order the library writes them
Bytes dataset_messages(bool integer, size_t n, size_t nbytes, const std::string& unit,
                       const std::string& desc, uint32_t now, uint64_t data_addr) {
    Bytes space = {1, 1, 1, 0, 0, 0, 0, 0};
    put<uint64_t>(space, n), put<uint64_t>(space, n);
    const Bytes fill = {2, 2, 2, 1, 0, 0, 0, 0};
    Bytes       layout = {3, 1};
    put<uint64_t>(layout, data_addr), put<uint64_t>(layout, nbytes);
    Bytes mtime = {1, 0, 0, 0};
    put<uint32_t>(mtime, now);
    Bytes m = message(kMsgDataspace, space);
    for (const Bytes& x : {message(kMsgDatatype, integer ? dt_i32() : dt_f64(), 1),
                           message(kMsgFill, fill, 1), message(kMsgLayout, layout),
                           message(kMsgMtime, mtime), attribute("Variable", desc),
                           attribute("units", unit)})
        put_bytes(m, x.data(), x.size());
    return m;
}

std::string strip(const std::string& name) { return name[0] == '/' ? name.substr(1) : name; }

} // namespace

void Writer::table(const std::string& name, const double* v, size_t n, const std::string& unit,
                   const std::string& description) {
    Item it{false, {}, unit, description};
    it.raw.reserve(8 * n);
    for (size_t i = 0; i < n; i++) {
        uint64_t bits;
        std::memcpy(&bits, v + i, 8);
        put<uint64_t>(it.raw, bits);
    }
    items_[strip(name)] = std::move(it);
}
void Writer::table_i32(const std::string& name, const int32_t* v, size_t n, const std::string& unit,
                       const std::string& description) {
    Item it{true, {}, unit, description};
    it.raw.reserve(4 * n);
    for (size_t i = 0; i < n; i++)
        put<uint32_t>(it.raw, (uint32_t)v[i]);
    items_[strip(name)] = std::move(it);
}
void Writer::value(const std::string& name, double v, const std::string& unit,
                   const std::string& description) {
    table(name, &v, 1, unit, description);
}
void Writer::value_i32(const std::string& name, int32_t v, const std::string& unit,
                       const std::string& description) {
    table_i32(name, &v, 1, unit, description);
}

bool Writer::close(const std::string& path, std::string* err) {
    std::vector<std::string> names;
    for (const auto& kv : items_)
        names.push_back(kv.first);
    if (names.size() > (size_t)kSnodCap * kBtreeCap) {
        *err = "more datasets than one B-tree node holds";
        return false;
    }
    // local heap: the empty name at 0, then every name (null-terminated, 8-byte aligned), then
    // one free block
    Bytes                         heap(8, 0);
    std::map<std::string, size_t> name_off;
    for (const auto& n : names) {
        name_off[n] = heap.size();
        put_bytes(heap, n.data(), n.size());
        heap.push_back(0);
        pad8(heap);
    }
    const size_t free_off = heap.size();
    put<uint64_t>(heap, 1), put<uint64_t>(heap, 16);
    const size_t nsnod      = std::max<size_t>(1, (names.size() + kSnodCap - 1) / kSnodCap);
    const size_t snod_size  = 8 + kSnodCap * 40;
    const size_t btree_size = 24 + 8 * (2 * kInternalK + 1) + 8 * (2 * kInternalK);
    // addresses: superblock, root object header, B-tree, heap header, heap data, symbol-table
    // nodes, then per dataset its object header and its data
    const size_t a_root = 96, a_btree = a_root + 16 + 24, a_heap = a_btree + btree_size;
    const size_t a_heapdata = a_heap + 32, a_snod = a_heapdata + heap.size();
    size_t       pos = a_snod + nsnod * snod_size;
    const uint32_t now = (uint32_t)(std::time(nullptr) & 0xFFFFFFFF);
    struct Obj {
        size_t addr, data_addr;
        Bytes  ohdr;
        const Bytes* raw;
    };
    std::vector<Obj>              objects;
    std::map<std::string, size_t> addr_of;
    for (const auto& n : names) {
        const Item&  it     = items_[n];
        const size_t count  = it.raw.size() / (it.integer ? 4 : 8);
        const size_t hdr    = 16 + dataset_messages(it.integer, count, it.raw.size(), it.unit,
                                                    it.description, now, 0).size();
        const size_t daddr  = pos + hdr;
        const Bytes  msgs   = dataset_messages(it.integer, count, it.raw.size(), it.unit,
                                               it.description, now, daddr);
        Bytes        ohdr;
        put<uint8_t>(ohdr, 1), put<uint8_t>(ohdr, 0);
        put<uint16_t>(ohdr, 7);
        put<uint32_t>(ohdr, 1);
        put<uint32_t>(ohdr, (uint32_t)msgs.size());
        put<uint32_t>(ohdr, 0);
        put_bytes(ohdr, msgs.data(), msgs.size());
        addr_of[n] = pos;
        objects.push_back({pos, daddr, std::move(ohdr), &it.raw});
        pos = daddr + it.raw.size();
        pos += (8 - pos % 8) % 8;
    }
    const size_t eof = pos;
    Bytes        out(eof, 0);
    // superblock v0 with the root group's symbol-table entry (cache type 1: B-tree, heap)
    std::memcpy(out.data(), kSignature, 8);
    const uint8_t versions[8] = {0, 0, 0, 0, 0, 8, 8, 0};
    std::memcpy(out.data() + 8, versions, 8);
    poke<uint16_t>(out, 16, kLeafK), poke<uint16_t>(out, 18, kInternalK);
    poke<uint32_t>(out, 20, 0);
    poke<uint64_t>(out, 24, 0), poke<uint64_t>(out, 32, kUndef), poke<uint64_t>(out, 40, eof);
    poke<uint64_t>(out, 48, kUndef);
    poke<uint64_t>(out, 56, 0), poke<uint64_t>(out, 64, a_root);
    poke<uint32_t>(out, 72, 1), poke<uint32_t>(out, 76, 0);
    poke<uint64_t>(out, 80, a_btree), poke<uint64_t>(out, 88, a_heap);
    // root object header: one symbol-table message
    {
        Bytes st;
        put<uint64_t>(st, a_btree), put<uint64_t>(st, a_heap);
        const Bytes m = message(kMsgSymtab, st);
        Bytes       root;
        put<uint8_t>(root, 1), put<uint8_t>(root, 0);
        put<uint16_t>(root, 1);
        put<uint32_t>(root, 1), put<uint32_t>(root, (uint32_t)m.size()), put<uint32_t>(root, 0);
        put_bytes(root, m.data(), m.size());
        std::memcpy(out.data() + a_root, root.data(), root.size());
    }
    // symbol-table nodes and the B-tree over them; key i + 1 = the last name of child i
    std::vector<uint64_t> keys = {0}, kids;
    for (size_t k = 0; k < nsnod; k++) {
        const size_t first = k * kSnodCap, last = std::min(names.size(), first + kSnodCap);
        const size_t a = a_snod + k * snod_size;
        Bytes        node = {'S', 'N', 'O', 'D', 1, 0};
        put<uint16_t>(node, (uint16_t)(last - first));
        for (size_t i = first; i < last; i++) {
            put<uint64_t>(node, name_off[names[i]]), put<uint64_t>(node, addr_of[names[i]]);
            put<uint32_t>(node, 0), put<uint32_t>(node, 0);
            node.insert(node.end(), 16, 0);
        }
        std::memcpy(out.data() + a, node.data(), node.size());
        kids.push_back(a);
        keys.push_back(last > first ? name_off[names[last - 1]] : 0);
    }
    {
        Bytes bt = {'T', 'R', 'E', 'E', 0, 0};
        put<uint16_t>(bt, (uint16_t)kids.size());
        put<uint64_t>(bt, kUndef), put<uint64_t>(bt, kUndef);
        for (size_t i = 0; i < kids.size(); i++)
            put<uint64_t>(bt, keys[i]), put<uint64_t>(bt, kids[i]);
        put<uint64_t>(bt, keys[kids.size()]);
        std::memcpy(out.data() + a_btree, bt.data(), bt.size());
    }
    // local heap header and data
    {
        Bytes h = {'H', 'E', 'A', 'P', 0, 0, 0, 0};
        put<uint64_t>(h, heap.size()), put<uint64_t>(h, free_off), put<uint64_t>(h, a_heapdata);
        std::memcpy(out.data() + a_heap, h.data(), h.size());
        std::memcpy(out.data() + a_heapdata, heap.data(), heap.size());
    }
    for (const Obj& o : objects) {
        std::memcpy(out.data() + o.addr, o.ohdr.data(), o.ohdr.size());
        if (!o.raw->empty())
            std::memcpy(out.data() + o.data_addr, o.raw->data(), o.raw->size());
    }
    const std::string tmp = path + ".tmp";
    {
        std::ofstream f(tmp, std::ios::binary | std::ios::trunc);
        if (!f || !f.write((const char*)out.data(), (std::streamsize)out.size())) {
            *err = "cannot write " + tmp;
            return false;
        }
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) {
        *err = "cannot rename " + tmp + " to " + path;
        return false;
    }
    return true;
}

// ---------------------------------------------------------------------------------------------
// Reader
// ---------------------------------------------------------------------------------------------
namespace {

struct Fail {
    std::string what;
};

struct File {
    Bytes d;
    template<class T>
    T u(uint64_t off) const {
        if (off + sizeof(T) > d.size())
            throw Fail{"read past the end of the file"};
        uint64_t v = 0;
        for (size_t i = 0; i < sizeof(T); i++)
            v |= (uint64_t)d[off + i] << (8 * i);
        return (T)v;
    }
    std::string cstr(uint64_t off) const {
        std::string s;
        while (off < d.size() && d[off])
            s.push_back((char)d[off++]);
        return s;
    }
    bool tag(uint64_t off, const char* t) const {
        return off + 4 <= d.size() && std::memcmp(d.data() + off, t, 4) == 0;
    }
    // (type, body offset, body size) of every message of the object header v1 at addr,
    // continuation blocks followed
    struct Msg {
        uint16_t type;
        uint64_t off, size;
    };
    std::vector<Msg> messages(uint64_t addr) const {
        if (u<uint8_t>(addr) != 1)
            throw Fail{"object header version other than 1"};
        const uint16_t nmsgs = u<uint16_t>(addr + 2);
        std::vector<std::pair<uint64_t, uint64_t>> chunks = {{addr + 16, u<uint32_t>(addr + 8)}};
        std::vector<Msg>                            out;
        while (!chunks.empty() && out.size() < nmsgs) {
            uint64_t p = chunks.front().first, end = p + chunks.front().second;
            chunks.erase(chunks.begin());
            while (p + 8 <= end && out.size() < nmsgs) {
                const uint16_t t = u<uint16_t>(p), sz = u<uint16_t>(p + 2);
                if (p + 8 + sz > d.size())
                    throw Fail{"message past the end of the file"};
                if (t == kMsgContinuation)
                    chunks.push_back({u<uint64_t>(p + 8), u<uint64_t>(p + 16)});
                out.push_back({t, p + 8, sz});
                p += 8 + sz;
            }
        }
        return out;
    }
    void walk(uint64_t node, uint64_t heap_data, std::map<std::string, uint64_t>& out,
              int depth) const {
        if (depth > 64 || !tag(node, "TREE") || u<uint8_t>(node + 4) != 0)
            throw Fail{"bad group B-tree node"};
        const int level = u<uint8_t>(node + 5), used = u<uint16_t>(node + 6);
        uint64_t  p = node + 24;
        for (int i = 0; i < used; i++, p += 16) {
            const uint64_t child = u<uint64_t>(p + 8);
            if (level > 0) {
                walk(child, heap_data, out, depth + 1);
                continue;
            }
            if (!tag(child, "SNOD"))
                throw Fail{"bad symbol-table node"};
            const int nsym = u<uint16_t>(child + 6);
            for (int s = 0; s < nsym; s++) {
                const uint64_t e = child + 8 + 40 * (uint64_t)s;
                out[cstr(heap_data + u<uint64_t>(e))] = u<uint64_t>(e + 8);
            }
        }
    }
};

// a datatype message: class (0 fixed-point, 1 floating-point, 3 string), size, signedness, order
struct Type {
    int  cls, size;
    bool is_signed, big;
};
Type datatype(const File& F, uint64_t b) {
    Type t;
    t.cls       = F.u<uint8_t>(b) & 0x0F;
    const int f = F.u<uint8_t>(b + 1);
    t.size      = (int)F.u<uint32_t>(b + 4);
    t.big       = (t.cls == 0 || t.cls == 1) && (f & 1);
    t.is_signed = t.cls == 0 && (f & 8);
    if (t.cls != 0 && t.cls != 1 && t.cls != 3)
        throw Fail{"datatype class " + std::to_string(t.cls) + " not read"};
    if ((t.cls == 0 && t.size != 1 && t.size != 2 && t.size != 4 && t.size != 8)
        || (t.cls == 1 && t.size != 4 && t.size != 8))
        throw Fail{"numeric datatype size not read"};
    return t;
}
std::vector<uint64_t> dataspace(const File& F, uint64_t b) {
    const int ver = F.u<uint8_t>(b), rank = F.u<uint8_t>(b + 1);
    std::vector<uint64_t> shape;
    if (ver == 1) {
        for (int i = 0; i < rank; i++)
            shape.push_back(F.u<uint64_t>(b + 8 + 8 * i));
    }
    else if (ver == 2) {
        if (F.u<uint8_t>(b + 3) != 0)
            for (int i = 0; i < rank; i++)
                shape.push_back(F.u<uint64_t>(b + 4 + 8 * i));
    }
    else
        throw Fail{"dataspace version " + std::to_string(ver)};
    return shape;
}
double element(const File& F, const Type& t, uint64_t at) {
    uint64_t v = 0;
    for (int i = 0; i < t.size; i++) {
        const int k = t.big ? t.size - 1 - i : i;
        v |= (uint64_t)F.u<uint8_t>(at + k) << (8 * i);
    }
    if (t.cls == 1) {
        if (t.size == 8) {
            double x;
            std::memcpy(&x, &v, 8);
            return x;
        }
        const uint32_t w = (uint32_t)v;
        float          x;
        std::memcpy(&x, &w, 4);
        return x;
    }
    if (t.is_signed && t.size < 8 && (v >> (8 * t.size - 1)) & 1)
        v |= ~0ull << (8 * t.size);
    return t.is_signed ? (double)(int64_t)v : (double)v;
}
std::string text(const File& F, const Type& t, uint64_t at) {
    std::string s;
    for (int i = 0; i < t.size && F.u<uint8_t>(at + i); i++)
        s.push_back((char)F.u<uint8_t>(at + i));
    return s;
}
uint64_t count_of(const std::vector<uint64_t>& shape) {
    uint64_t n = 1;
    for (uint64_t s : shape)
        n *= s;
    return n;
}

void attribute(const File& F, uint64_t b, Dataset& ds) {
    const int ver = F.u<uint8_t>(b);
    const int nsz = F.u<uint16_t>(b + 2), tsz = F.u<uint16_t>(b + 4), ssz = F.u<uint16_t>(b + 6);
    auto      r8  = [](int n) { return (uint64_t)(n + (8 - n % 8) % 8); };
    uint64_t  p;
    std::string name;
    Type        t;
    std::vector<uint64_t> shape;
    if (ver == 1) {
        p    = b + 8;
        name = F.cstr(p);
        p += r8(nsz);
        t = datatype(F, p);
        p += r8(tsz);
        shape = dataspace(F, p);
        p += r8(ssz);
    }
    else if (ver == 2 || ver == 3) {
        p    = b + 8 + (ver == 3 ? 1 : 0);
        name = F.cstr(p);
        p += nsz;
        t = datatype(F, p);
        p += tsz;
        shape = dataspace(F, p);
        p += ssz;
    }
    else
        throw Fail{"attribute version " + std::to_string(ver)};
    if (t.cls == 3)
        ds.attrs[name] = text(F, t, p);
}

Dataset dataset(const File& F, uint64_t addr) {
    Dataset ds;
    bool    have_space = false, have_type = false, have_data = false, compact = false;
    Type    t{};
    uint64_t data_at = 0;
    for (const File::Msg& m : F.messages(addr)) {
        if (m.type == kMsgDataspace) {
            ds.shape   = dataspace(F, m.off);
            have_space = true;
        }
        else if (m.type == kMsgDatatype) {
            t         = datatype(F, m.off);
            have_type = true;
        }
        else if (m.type == kMsgLayout) {
            if (F.u<uint8_t>(m.off) != 3)
                throw Fail{"layout version other than 3"};
            const int cls = F.u<uint8_t>(m.off + 1);
            if (cls == 1)
                data_at = F.u<uint64_t>(m.off + 2);
            else if (cls == 0) {
                data_at = m.off + 4;
                compact = true;
            }
            else
                throw Fail{"chunked layout not read"};
            have_data = true;
        }
        else if (m.type == kMsgAttribute)
            attribute(F, m.off, ds);
    }
    if (!have_space || !have_type || !have_data)
        throw Fail{"object is not a dataset"};
    if (t.cls == 3)
        throw Fail{"string datasets not read"};
    (void)compact;
    ds.integer        = t.cls == 0;
    const uint64_t n  = count_of(ds.shape);
    ds.values.resize(n, 0.0);
    if (data_at != kUndef)
        for (uint64_t i = 0; i < n; i++)
            ds.values[i] = element(F, t, data_at + i * t.size);
    return ds;
}

} // namespace

bool read(const std::string& path, std::map<std::string, Dataset>& out, std::string* err) {
    File F;
    {
        std::ifstream f(path, std::ios::binary);
        if (!f) {
            *err = "cannot open " + path;
            return false;
        }
        F.d.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    }
    try {
        if (F.d.size() < 96 || std::memcmp(F.d.data(), kSignature, 8) != 0)
            throw Fail{"not an HDF5 file (signature)"};
        if (F.d[8] != 0)
            throw Fail{"superblock version other than 0"};
        if (F.d[13] != 8 || F.d[14] != 8)
            throw Fail{"sizes of offsets/lengths other than 8"};
        const uint64_t root = F.u<uint64_t>(64);
        uint64_t       btree = kUndef, heap = kUndef;
        for (const File::Msg& m : F.messages(root))
            if (m.type == kMsgSymtab) {
                btree = F.u<uint64_t>(m.off);
                heap  = F.u<uint64_t>(m.off + 8);
            }
        if (btree == kUndef)
            throw Fail{"root group without a symbol table"};
        if (!F.tag(heap, "HEAP"))
            throw Fail{"bad local heap"};
        std::map<std::string, uint64_t> entries;
        F.walk(btree, F.u<uint64_t>(heap + 24), entries, 0);
        out.clear();
        for (const auto& kv : entries)
            out[kv.first] = dataset(F, kv.second);
    }
    catch (const Fail& e) {
        *err = path + ": " + e.what;
        return false;
    }
    return true;
}

} // namespace thorx_h5
