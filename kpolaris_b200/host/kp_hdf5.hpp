// kp_hdf5.hpp -- a minimal HDF5 file writer for the image tool's output
// (the kpolaris_image v1 layout, tools/kpolaris_model_image.cpp:4284-4840 and
// docs/hdf5_schema.md in the reference).  No HDF5 library is available to
// this build, so the subset of the HDF5 file format the image schema needs
// is written directly from the format specification:
//   * superblock version 2 (8-byte offsets and lengths);
//   * version-2 object headers ("OHDR", one chunk, Jenkins lookup3 checksum);
//   * groups with compact link storage: a Link Info message (no fractal
//     heap), a Group Info message and one hard-link Link message per child;
//   * datasets with a version-2 Dataspace, a Datatype, a version-3 Fill Value
//     (late allocation, none defined) and a contiguous version-3 Data Layout;
//   * scalar attributes (version-3 Attribute messages) of IEEE little-endian
//     float64, little-endian int32 or null-terminated fixed-length ASCII
//     strings.
// Objects are laid out as: superblock, every object header in depth-first
// order, then every dataset's raw data (8-byte aligned).  Links and
// attributes keep insertion order.
#pragma once

#include <cstdint>
#include <cstring>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace kph5 {

// Bob Jenkins' lookup3 hashlittle (public domain, 2006), byte-at-a-time form:
// the checksum of HDF5's version-2 metadata with initval 0.
inline uint32_t lookup3(const uint8_t* k, size_t length, uint32_t initval) {
    auto rot = [](uint32_t x, int r) { return (x << r) | (x >> (32 - r)); };
    uint32_t a, b, c;
    a = b = c = 0xdeadbeefu + uint32_t(length) + initval;
    while (length > 12) {
        a += k[0] + (uint32_t(k[1]) << 8) + (uint32_t(k[2]) << 16) + (uint32_t(k[3]) << 24);
        b += k[4] + (uint32_t(k[5]) << 8) + (uint32_t(k[6]) << 16) + (uint32_t(k[7]) << 24);
        c += k[8] + (uint32_t(k[9]) << 8) + (uint32_t(k[10]) << 16) + (uint32_t(k[11]) << 24);
        a -= c; a ^= rot(c, 4);  c += b;
        b -= a; b ^= rot(a, 6);  a += c;
        c -= b; c ^= rot(b, 8);  b += a;
        a -= c; a ^= rot(c, 16); c += b;
        b -= a; b ^= rot(a, 19); a += c;
        c -= b; c ^= rot(b, 4);  b += a;
        length -= 12;
        k += 12;
    }
    switch (length) {
    case 12: c += uint32_t(k[11]) << 24; [[fallthrough]];
    case 11: c += uint32_t(k[10]) << 16; [[fallthrough]];
    case 10: c += uint32_t(k[9]) << 8; [[fallthrough]];
    case 9: c += k[8]; [[fallthrough]];
    case 8: b += uint32_t(k[7]) << 24; [[fallthrough]];
    case 7: b += uint32_t(k[6]) << 16; [[fallthrough]];
    case 6: b += uint32_t(k[5]) << 8; [[fallthrough]];
    case 5: b += k[4]; [[fallthrough]];
    case 4: a += uint32_t(k[3]) << 24; [[fallthrough]];
    case 3: a += uint32_t(k[2]) << 16; [[fallthrough]];
    case 2: a += uint32_t(k[1]) << 8; [[fallthrough]];
    case 1: a += k[0]; break;
    case 0: return c;
    }
    c ^= b; c -= rot(b, 14);
    a ^= c; a -= rot(c, 11);
    b ^= a; b -= rot(a, 25);
    c ^= b; c -= rot(b, 16);
    a ^= c; a -= rot(c, 4);
    b ^= a; b -= rot(a, 14);
    c ^= b; c -= rot(b, 24);
    return c;
}

enum class Kind { F64, I32, Str };

struct Attribute {
    std::string name;
    Kind kind;
    double f = 0.0;
    int32_t i = 0;
    std::string s;
};

struct Dataset {
    std::string name;
    Kind kind;  // F64 or I32
    std::vector<uint64_t> dims;
    std::vector<uint8_t> bytes;
    std::vector<Attribute> attrs;
    uint64_t header_addr = 0, data_addr = 0;
};

class Group {
public:
    explicit Group(std::string name = "") : name_(std::move(name)) {}

    Group& group(const std::string& name) {
        check_new(name);
        order_.push_back({0, groups_.size()});
        groups_.push_back(std::make_unique<Group>(name));
        return *groups_.back();
    }
    void attr(const std::string& name, double v) { add({name, Kind::F64, v, 0, {}}); }
    void attr(const std::string& name, int v) { add({name, Kind::I32, 0.0, int32_t(v), {}}); }
    void attr(const std::string& name, const std::string& v) { add({name, Kind::Str, 0.0, 0, v}); }
    void attr(const std::string& name, const char* v) { attr(name, std::string(v)); }
    void dataset(const std::string& name, const std::vector<uint64_t>& dims, const double* data) {
        put(name, Kind::F64, dims, data, sizeof(double));
    }
    void dataset(const std::string& name, const std::vector<uint64_t>& dims, const int32_t* data) {
        put(name, Kind::I32, dims, data, sizeof(int32_t));
    }

private:
    friend class File;
    struct Link {
        int is_dataset;
        size_t index;
    };
    void check_new(const std::string& name) {
        if (name.empty() || name.size() > 255 || name.find('/') != std::string::npos)
            throw std::runtime_error("HDF5 link name not writable: '" + name + "'");
        for (const auto& g : groups_)
            if (g->name_ == name) throw std::runtime_error("HDF5 link exists: " + name);
        for (const auto& d : datasets_)
            if (d.name == name) throw std::runtime_error("HDF5 link exists: " + name);
    }
    void add(const Attribute& a) {
        for (auto& x : attrs_)
            if (x.name == a.name) {
                x = a;  // the latest value of a repeated attribute
                return;
            }
        attrs_.push_back(a);
    }
    void put(const std::string& name, Kind kind, const std::vector<uint64_t>& dims, const void* data, size_t esize) {
        check_new(name);
        Dataset d;
        d.name = name;
        d.kind = kind;
        d.dims = dims;
        uint64_t n = 1;
        for (uint64_t v : dims) n *= v;
        d.bytes.resize(size_t(n) * esize);
        if (n) std::memcpy(d.bytes.data(), data, d.bytes.size());
        order_.push_back({1, datasets_.size()});
        datasets_.push_back(std::move(d));
    }

    std::string name_;
    std::vector<Attribute> attrs_;
    std::vector<std::unique_ptr<Group>> groups_;
    std::vector<Dataset> datasets_;
    std::vector<Link> order_;
    uint64_t header_addr_ = 0;
};

class File {
public:
    Group& root() { return root_; }

    void write(const std::string& path) {
        // pass 1: header sizes and addresses, then raw data addresses
        uint64_t at = kSuperblock;
        place_headers(root_, at);
        at = (at + 7) & ~uint64_t(7);
        place_data(root_, at);
        const uint64_t eof = at;
        // pass 2: bytes
        std::vector<uint8_t> out;
        out.reserve(size_t(eof));
        superblock(out, eof);
        emit_headers(root_, out);
        while (out.size() % 8) out.push_back(0);
        emit_data(root_, out);
        if (out.size() != eof) throw std::runtime_error("HDF5 writer: layout size mismatch");
        std::ofstream f(path, std::ios::binary | std::ios::trunc);
        if (!f) throw std::runtime_error("failed to open output: " + path);
        f.write(reinterpret_cast<const char*>(out.data()), std::streamsize(out.size()));
        if (!f) throw std::runtime_error("failed writing output: " + path);
    }

private:
    static constexpr uint64_t kSuperblock = 48;
    static constexpr uint64_t kUndef = ~uint64_t(0);

    // --- byte helpers
    static void u8(std::vector<uint8_t>& b, unsigned v) { b.push_back(uint8_t(v)); }
    static void le(std::vector<uint8_t>& b, uint64_t v, int n) {
        for (int k = 0; k < n; ++k) b.push_back(uint8_t(v >> (8 * k)));
    }
    static void bytes(std::vector<uint8_t>& b, const void* p, size_t n) {
        const uint8_t* c = static_cast<const uint8_t*>(p);
        b.insert(b.end(), c, c + n);
    }

    // --- datatype and dataspace encodings
    static std::vector<uint8_t> datatype(Kind k, size_t strsize = 0) {
        std::vector<uint8_t> t;
        if (k == Kind::F64) {
            u8(t, 0x11);                        // version 1, floating point
            u8(t, 0x20); u8(t, 63); u8(t, 0);   // little-endian, implied mantissa msb, sign bit 63
            le(t, 8, 4);                        // size
            le(t, 0, 2); le(t, 64, 2);          // bit offset, precision
            u8(t, 52); u8(t, 11); u8(t, 0); u8(t, 52);  // exponent location/size, mantissa location/size
            le(t, 1023, 4);                     // exponent bias
        } else if (k == Kind::I32) {
            u8(t, 0x10);                        // version 1, fixed point
            u8(t, 0x08); u8(t, 0); u8(t, 0);    // little-endian, signed
            le(t, 4, 4);
            le(t, 0, 2); le(t, 32, 2);
        } else {
            u8(t, 0x13);                        // version 1, string
            u8(t, 0x00); u8(t, 0); u8(t, 0);    // null-terminated, ASCII
            le(t, strsize, 4);
        }
        return t;
    }
    static std::vector<uint8_t> dataspace(const std::vector<uint64_t>& dims) {
        std::vector<uint8_t> s;
        u8(s, 2);                                // version 2
        u8(s, unsigned(dims.size()));            // rank
        u8(s, 0);                                // no maximum dimensions
        u8(s, dims.empty() ? 0 : 1);             // scalar or simple
        for (uint64_t d : dims) le(s, d, 8);
        return s;
    }

    // --- messages
    static void message(std::vector<uint8_t>& b, unsigned type, const std::vector<uint8_t>& data, unsigned flags = 0) {
        if (data.size() > 0xffff) throw std::runtime_error("HDF5 writer: header message too large");
        u8(b, type);
        le(b, data.size(), 2);
        u8(b, flags);
        bytes(b, data.data(), data.size());
    }
    static std::vector<uint8_t> attribute(const Attribute& a) {
        std::vector<uint8_t> m;
        const size_t ssize = a.kind == Kind::Str ? a.s.size() + 1 : 0;
        const std::vector<uint8_t> dt = datatype(a.kind, ssize);
        const std::vector<uint8_t> ds = dataspace({});
        u8(m, 3);                               // version 3
        u8(m, 0);                               // neither type nor space shared
        le(m, a.name.size() + 1, 2);
        le(m, dt.size(), 2);
        le(m, ds.size(), 2);
        u8(m, 0);                               // name encoding ASCII
        bytes(m, a.name.c_str(), a.name.size() + 1);
        bytes(m, dt.data(), dt.size());
        bytes(m, ds.data(), ds.size());
        if (a.kind == Kind::F64) {
            uint64_t v;
            std::memcpy(&v, &a.f, 8);
            le(m, v, 8);
        } else if (a.kind == Kind::I32) {
            le(m, uint32_t(a.i), 4);
        } else {
            bytes(m, a.s.c_str(), a.s.size() + 1);
        }
        return m;
    }
    // The messages of a group's object header (addresses of the children
    // must be placed before it is called for bytes).
    std::vector<uint8_t> group_messages(const Group& g) const {
        std::vector<uint8_t> b;
        std::vector<uint8_t> linfo;
        u8(linfo, 0); u8(linfo, 0);             // version 0, no creation order
        le(linfo, kUndef, 8);                   // no fractal heap: compact links
        le(linfo, kUndef, 8);                   // no name index
        message(b, 0x02, linfo);
        message(b, 0x0A, {0, 0});               // group info: version 0, defaults
        for (const auto& l : g.order_) {
            const std::string& name = l.is_dataset ? g.datasets_[l.index].name : g.groups_[l.index]->name_;
            const uint64_t addr = l.is_dataset ? g.datasets_[l.index].header_addr : g.groups_[l.index]->header_addr_;
            std::vector<uint8_t> link;
            u8(link, 1);                        // version 1
            u8(link, 0);                        // 1-byte name length, hard link, ASCII
            u8(link, unsigned(name.size()));
            bytes(link, name.data(), name.size());
            le(link, addr, 8);
            message(b, 0x06, link);
        }
        for (const auto& a : g.attrs_) message(b, 0x0C, attribute(a));
        return b;
    }
    static std::vector<uint8_t> dataset_messages(const Dataset& d) {
        std::vector<uint8_t> b;
        message(b, 0x01, dataspace(d.dims));
        message(b, 0x03, datatype(d.kind), 0x01);  // constant
        message(b, 0x05, {3, 0x0A});               // fill value v3: late allocation, written if set, none set
        std::vector<uint8_t> layout;
        u8(layout, 3);                             // version 3
        u8(layout, 1);                             // contiguous
        le(layout, d.data_addr, 8);
        le(layout, d.bytes.size(), 8);
        message(b, 0x08, layout);
        for (const auto& a : d.attrs) message(b, 0x0C, attribute(a));
        return b;
    }
    static uint64_t header_size(size_t messages) { return 4 + 1 + 1 + 4 + messages + 4; }
    static void object_header(std::vector<uint8_t>& out, const std::vector<uint8_t>& msgs) {
        const size_t start = out.size();
        bytes(out, "OHDR", 4);
        u8(out, 2);                                // version 2
        u8(out, 0x02);                             // chunk #0 size in 4 bytes; no times, no creation order
        le(out, msgs.size(), 4);
        bytes(out, msgs.data(), msgs.size());
        const uint32_t sum = lookup3(out.data() + start, out.size() - start, 0);
        le(out, sum, 4);
    }

    void place_headers(Group& g, uint64_t& at) {
        g.header_addr_ = at;
        at += header_size(group_messages(g).size());
        for (const auto& l : g.order_) {
            if (l.is_dataset) {
                Dataset& d = g.datasets_[l.index];
                d.header_addr = at;
                at += header_size(dataset_messages(d).size());
            } else {
                place_headers(*g.groups_[l.index], at);
            }
        }
    }
    void place_data(Group& g, uint64_t& at) {
        for (const auto& l : g.order_) {
            if (l.is_dataset) {
                Dataset& d = g.datasets_[l.index];
                d.data_addr = d.bytes.empty() ? kUndef : at;
                at += d.bytes.size();
                at = (at + 7) & ~uint64_t(7);
            } else {
                place_data(*g.groups_[l.index], at);
            }
        }
    }
    void superblock(std::vector<uint8_t>& out, uint64_t eof) const {
        const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
        bytes(out, sig, 8);
        u8(out, 2);                                // superblock version 2
        u8(out, 8);                                // size of offsets
        u8(out, 8);                                // size of lengths
        u8(out, 0);                                // file consistency flags
        le(out, 0, 8);                             // base address
        le(out, kUndef, 8);                        // no superblock extension
        le(out, eof, 8);                           // end of file address
        le(out, root_.header_addr_, 8);            // root group object header
        le(out, lookup3(out.data(), out.size(), 0), 4);
    }
    void emit_headers(const Group& g, std::vector<uint8_t>& out) const {
        if (out.size() != g.header_addr_) throw std::runtime_error("HDF5 writer: header address mismatch");
        object_header(out, group_messages(g));
        for (const auto& l : g.order_) {
            if (l.is_dataset) {
                const Dataset& d = g.datasets_[l.index];
                if (out.size() != d.header_addr) throw std::runtime_error("HDF5 writer: header address mismatch");
                object_header(out, dataset_messages(d));
            } else {
                emit_headers(*g.groups_[l.index], out);
            }
        }
    }
    void emit_data(const Group& g, std::vector<uint8_t>& out) const {
        for (const auto& l : g.order_) {
            if (l.is_dataset) {
                const Dataset& d = g.datasets_[l.index];
                if (!d.bytes.empty()) {
                    if (out.size() != d.data_addr) throw std::runtime_error("HDF5 writer: data address mismatch");
                    bytes(out, d.bytes.data(), d.bytes.size());
                }
                while (out.size() % 8) out.push_back(0);
            } else {
                emit_data(*g.groups_[l.index], out);
            }
        }
    }

    Group root_{""};
};

}  // namespace kph5
