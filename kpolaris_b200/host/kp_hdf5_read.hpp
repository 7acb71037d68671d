// kp_hdf5_read.hpp -- reads numeric datasets out of HDF5 files written by the
// HDF5 library, for the GRMHD dump loaders (iharm: src/grmhd/iharm_loader.cpp
// in the reference, which reads through the HDF5 C++ API).  No HDF5 library
// is available to this build, so the structures the library writes for such
// files are read directly from the HDF5 file format specification:
//   * superblock versions 0 and 1 (the library's default, "earliest" format)
//     and 2 and 3 ("latest"), with a user block before it;
//   * object headers version 1 (8-byte aligned messages, continuation
//     blocks) and version 2 ("OHDR"/"OCHK" chunks, lookup3 checksums);
//   * groups with a symbol table (version-1 B-tree of group nodes, "SNOD"
//     symbol nodes, local heap of names) or with compact link storage (Link
//     messages); dense link storage (fractal heap) is refused;
//   * datasets of IEEE float (32/64) or integer (8/16/32/64, either sign)
//     little-endian elements, with version 1/2 or version 1 Dataspace
//     messages, and compact, contiguous or chunked Data Layout messages
//     (versions 1-3; version 4 for compact, contiguous and the single-chunk
//     and implicit chunk indexes);
//   * chunks indexed by a version-1 B-tree (raw data nodes) and the filters
//     deflate and shuffle.
// Anything else raises kph5::FormatError naming what it met, so a file the
// subset does not cover is refused rather than misread.  Values are
// converted to the caller's type as the library's H5Dread conversion to a
// native type would (integers to float by value, doubles to float rounded to
// nearest).
#pragma once

#include <zlib.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "kp_hdf5.hpp"

namespace kph5 {

struct FormatError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

enum class ElemType { Int, UInt, Float, String, VarString, Other };

struct DatasetInfo {
    std::vector<uint64_t> dims;  // empty: scalar
    ElemType type = ElemType::Other;
    size_t elem = 0;
    int layout = -1;             // 0 compact, 1 contiguous, 2 chunked
    uint64_t addr = 0;           // contiguous data or chunk index address
    uint64_t size = 0;           // contiguous data bytes
    std::vector<uint8_t> compact;
    std::vector<uint64_t> chunk; // chunk dims in elements (rank entries)
    int chunk_index = 0;         // 0 v1 B-tree, 1 single chunk, 2 implicit
    uint64_t single_size = 0;    // single chunk: stored (filtered) bytes
    uint32_t single_mask = 0;
    struct Filter {
        uint16_t id;
        std::vector<uint32_t> values;
    };
    std::vector<Filter> filters;

    uint64_t count() const {
        uint64_t n = 1;
        for (uint64_t d : dims) n *= d;
        return n;
    }
};

class Reader {
public:
    explicit Reader(const std::string& path) : path_(path) {
        f_ = std::fopen(path.c_str(), "rb");
        if (!f_) throw FormatError("cannot open HDF5 file: " + path);
        std::fseek(f_, 0, SEEK_END);
        file_size_ = uint64_t(std::ftell(f_));
        try {
            superblock();
        } catch (...) {
            std::fclose(f_);
            throw;
        }
    }
    ~Reader() {
        if (f_) std::fclose(f_);
    }
    Reader(const Reader&) = delete;
    Reader& operator=(const Reader&) = delete;

    // True where every component of `path` ("/a/b/c") names a link.
    bool exists(const std::string& path) {
        uint64_t addr = 0;
        return resolve(path, addr);
    }

    DatasetInfo info(const std::string& path) {
        uint64_t addr = 0;
        if (!resolve(path, addr)) throw FormatError("HDF5 object not found: " + path);
        return dataset_info(addr, path);
    }

    // Every element of a numeric dataset, row-major, converted to T.
    template <class T>
    std::vector<T> read(const std::string& path) {
        const DatasetInfo d = info(path);
        return read<T>(d, path);
    }

    template <class T>
    std::vector<T> read(const DatasetInfo& d, const std::string& path) {
        if (d.type != ElemType::Int && d.type != ElemType::UInt && d.type != ElemType::Float)
            throw FormatError("HDF5 dataset " + path + " is not numeric");
        const std::vector<uint8_t> raw = raw_data(d, path);
        const uint64_t n = d.count();
        std::vector<T> out(static_cast<size_t>(n));
        for (uint64_t i = 0; i < n; ++i) out[size_t(i)] = convert<T>(raw.data() + i * d.elem, d);
        return out;
    }

    // An attribute of the object at `path` ("" or "/" for the root group):
    // numeric values row-major in `raw`, or the text of a fixed-length or
    // variable-length string in `text`.
    struct AttrValue {
        std::vector<uint64_t> dims;
        DatasetInfo type;
        std::vector<uint8_t> raw;
        std::string text;
        uint64_t count() const {
            uint64_t n = 1;
            for (uint64_t d : dims) n *= d;
            return n;
        }
    };

    bool has_attr(const std::string& path, const std::string& name) {
        AttrValue v;
        return find_attr(path, name, v, false);
    }

    AttrValue attr(const std::string& path, const std::string& name) {
        AttrValue v;
        if (!find_attr(path, name, v, true)) throw FormatError("HDF5 attribute not found: " + path + " " + name);
        return v;
    }

    template <class T>
    std::vector<T> attr_values(const std::string& path, const std::string& name) {
        const AttrValue v = attr(path, name);
        const DatasetInfo& d = v.type;
        if (d.type != ElemType::Int && d.type != ElemType::UInt && d.type != ElemType::Float)
            throw FormatError("HDF5 attribute " + name + " is not numeric");
        const uint64_t n = v.count();
        if (v.raw.size() < n * d.elem) throw FormatError("HDF5 attribute " + name + " truncated");
        std::vector<T> out(static_cast<size_t>(n));
        for (uint64_t i = 0; i < n; ++i) out[size_t(i)] = convert<T>(v.raw.data() + i * d.elem, d);
        return out;
    }

    std::string attr_string(const std::string& path, const std::string& name) {
        const AttrValue v = attr(path, name);
        if (v.type.type != ElemType::String && v.type.type != ElemType::VarString)
            throw FormatError("HDF5 attribute " + name + " is not a string");
        return v.text;
    }

    template <class T>
    T scalar(const std::string& path) {
        const std::vector<T> v = read<T>(path);
        if (v.size() != 1) throw FormatError("HDF5 dataset " + path + " is not a single value");
        return v[0];
    }

private:
    static constexpr uint64_t kUndef = ~uint64_t(0);
    std::string path_;
    std::FILE* f_ = nullptr;
    uint64_t file_size_ = 0;
    uint64_t base_ = 0;
    uint64_t root_ = 0;
    int so_ = 8;  // size of offsets
    int sl_ = 8;  // size of lengths

    struct Msg {
        uint16_t type;
        uint8_t flags;
        std::vector<uint8_t> data;
    };

    // -- file access ---------------------------------------------------------
    std::vector<uint8_t> bytes_at(uint64_t abs, uint64_t n) {
        if (abs > file_size_ || n > file_size_ - abs)
            throw FormatError("HDF5 read beyond the end of " + path_);
        std::vector<uint8_t> b(static_cast<size_t>(n));
        if (n == 0) return b;
        if (std::fseek(f_, long(abs), SEEK_SET) != 0 || std::fread(b.data(), 1, size_t(n), f_) != size_t(n))
            throw FormatError("HDF5 read failed in " + path_);
        return b;
    }
    std::vector<uint8_t> bytes(uint64_t addr, uint64_t n) {
        if (addr == kUndef) throw FormatError("HDF5 undefined address");
        return bytes_at(base_ + addr, n);
    }
    static uint64_t le(const uint8_t* p, int n) {
        uint64_t v = 0;
        for (int i = n - 1; i >= 0; --i) v = (v << 8) | p[i];
        return v;
    }
    uint64_t offset(const uint8_t* p) const {
        const uint64_t v = le(p, so_);
        return (so_ < 8 && v == (uint64_t(1) << (8 * so_)) - 1) ? kUndef : v;
    }
    uint64_t length(const uint8_t* p) const { return le(p, sl_); }

    struct Cursor {
        const std::vector<uint8_t>& b;
        size_t p;
        const uint8_t* need(size_t n) {
            if (p + n > b.size()) throw FormatError("HDF5 message truncated");
            const uint8_t* q = b.data() + p;
            p += n;
            return q;
        }
        uint64_t u(int n) { return le(need(size_t(n)), n); }
    };

    // -- superblock ----------------------------------------------------------
    void superblock() {
        static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
        uint64_t at = 0;
        for (;;) {
            if (at + 8 > file_size_) throw FormatError("not an HDF5 file: " + path_);
            const std::vector<uint8_t> s = bytes_at(at, 8);
            if (std::memcmp(s.data(), sig, 8) == 0) break;
            at = at == 0 ? 512 : at * 2;
        }
        const std::vector<uint8_t> h = bytes_at(at, std::min<uint64_t>(file_size_ - at, 256));
        if (h.size() < 12) throw FormatError("HDF5 superblock truncated");
        const int version = h[8];
        if (version == 0 || version == 1) {
            so_ = h[13];
            sl_ = h[14];
            check_sizes();
            size_t p = 24 + (version == 1 ? 4 : 0);
            if (h.size() < p + 4 * size_t(so_) + 2 * size_t(so_)) throw FormatError("HDF5 superblock truncated");
            base_ = le(&h[p], so_);
            p += 4 * size_t(so_);  // base, free space, end of file, driver information
            // root group symbol table entry: link name offset, object header address
            root_ = le(&h[p + size_t(so_)], so_);
        } else if (version == 2 || version == 3) {
            so_ = h[9];
            sl_ = h[10];
            check_sizes();
            const size_t p = 12;
            const size_t end = p + 4 * size_t(so_);
            if (h.size() < end + 4) throw FormatError("HDF5 superblock truncated");
            if (lookup3(h.data(), end, 0) != uint32_t(le(&h[end], 4)))
                throw FormatError("HDF5 superblock checksum mismatch");
            base_ = le(&h[p], so_);
            root_ = le(&h[p + 3 * size_t(so_)], so_);
        } else {
            throw FormatError("HDF5 superblock version " + std::to_string(version) + " is not supported");
        }
    }
    void check_sizes() const {
        if ((so_ != 4 && so_ != 8) || (sl_ != 4 && sl_ != 8))
            throw FormatError("HDF5 offset/length sizes other than 4 or 8 bytes");
    }

    // -- object headers ------------------------------------------------------
    std::vector<Msg> header(uint64_t addr) {
        std::vector<Msg> out;
        const std::vector<uint8_t> pre = bytes(addr, 16);
        if (std::memcmp(pre.data(), "OHDR", 4) == 0) {
            const int flags = pre[5];
            if (pre[4] != 2) throw FormatError("HDF5 object header version " + std::to_string(pre[4]));
            size_t p = 6 + ((flags & 0x20) ? 16 : 0) + ((flags & 0x10) ? 4 : 0);
            const int w = 1 << (flags & 0x03);
            const std::vector<uint8_t> pre2 = bytes(addr, p + size_t(w));
            const uint64_t chunk = le(&pre2[p], w);
            p += size_t(w);
            const std::vector<uint8_t> blk = bytes(addr, p + chunk + 4);
            if (lookup3(blk.data(), p + chunk, 0) != uint32_t(le(&blk[p + chunk], 4)))
                throw FormatError("HDF5 object header checksum mismatch");
            v2_messages(blk, p, p + chunk, flags, out);
        } else {
            if (pre[0] != 1) throw FormatError("HDF5 object header version " + std::to_string(pre[0]));
            const uint64_t size = le(&pre[8], 4);
            const std::vector<uint8_t> blk = bytes(addr + 16, size);
            v1_messages(blk, 0, blk.size(), out);
        }
        // continuation blocks (appended to `out` as they are read)
        for (size_t i = 0; i < out.size(); ++i) {
            if (out[i].type != 0x10) continue;
            Cursor c{out[i].data, 0};
            const uint64_t caddr = offset(c.need(size_t(so_)));
            const uint64_t clen = length(c.need(size_t(sl_)));
            const std::vector<uint8_t> blk = bytes(caddr, clen);
            if (blk.size() >= 4 && std::memcmp(blk.data(), "OCHK", 4) == 0) {
                if (clen < 8 || lookup3(blk.data(), size_t(clen) - 4, 0) != uint32_t(le(&blk[size_t(clen) - 4], 4)))
                    throw FormatError("HDF5 continuation chunk checksum mismatch");
                const int flags = bytes(addr, 6)[5];
                v2_messages(blk, 4, size_t(clen) - 4, flags, out);
            } else {
                v1_messages(blk, 0, blk.size(), out);
            }
        }
        return out;
    }
    static void v1_messages(const std::vector<uint8_t>& b, size_t p, size_t end, std::vector<Msg>& out) {
        while (p + 8 <= end) {
            Msg m;
            m.type = uint16_t(le(&b[p], 2));
            const size_t n = size_t(le(&b[p + 2], 2));
            m.flags = b[p + 4];
            p += 8;
            if (p + n > end) throw FormatError("HDF5 header message overruns its block");
            m.data.assign(b.begin() + long(p), b.begin() + long(p + n));
            p += n;
            if (m.type != 0) out.push_back(std::move(m));
        }
    }
    static void v2_messages(const std::vector<uint8_t>& b, size_t p, size_t end, int hflags,
                            std::vector<Msg>& out) {
        const size_t hdr = (hflags & 0x04) ? 6 : 4;
        while (p + hdr <= end) {
            Msg m;
            m.type = b[p];
            const size_t n = size_t(le(&b[p + 1], 2));
            m.flags = b[p + 3];
            p += hdr;
            if (p + n > end) throw FormatError("HDF5 header message overruns its chunk");
            m.data.assign(b.begin() + long(p), b.begin() + long(p + n));
            p += n;
            if (m.type != 0) out.push_back(std::move(m));
        }
    }
    static void refuse_shared(const Msg& m) {
        if (m.flags & 0x02) throw FormatError("HDF5 shared header messages are not supported");
    }

    // -- groups --------------------------------------------------------------
    bool resolve(const std::string& path, uint64_t& addr) {
        addr = root_;
        size_t i = 0;
        while (i < path.size()) {
            while (i < path.size() && path[i] == '/') ++i;
            if (i >= path.size()) break;
            size_t j = path.find('/', i);
            if (j == std::string::npos) j = path.size();
            if (!child(addr, path.substr(i, j - i), addr)) return false;
            i = j;
        }
        return true;
    }

    bool child(uint64_t group, const std::string& name, uint64_t& out) {
        const std::vector<Msg> msgs = header(group);
        bool is_group = false;
        for (const Msg& m : msgs) {
            if (m.type == 0x11) {  // symbol table
                is_group = true;
                Cursor c{m.data, 0};
                const uint64_t btree = offset(c.need(size_t(so_)));
                const uint64_t heap = offset(c.need(size_t(so_)));
                const std::vector<uint8_t> names = local_heap(heap);
                if (symbol_lookup(btree, names, name, out, 0)) return true;
            } else if (m.type == 0x02) {  // link info
                is_group = true;
                Cursor c{m.data, 0};
                if (c.u(1) != 0) throw FormatError("HDF5 link info version");
                const int flags = int(c.u(1));
                if (flags & 0x01) c.need(8);
                if (offset(c.need(size_t(so_))) != kUndef)
                    throw FormatError("HDF5 dense link storage (fractal heap) is not supported");
            } else if (m.type == 0x06) {  // link
                is_group = true;
                Cursor c{m.data, 0};
                if (c.u(1) != 1) throw FormatError("HDF5 link message version");
                const int flags = int(c.u(1));
                int ltype = 0;
                if (flags & 0x08) ltype = int(c.u(1));
                if (flags & 0x04) c.need(8);
                if (flags & 0x10) c.need(1);
                const uint64_t nlen = c.u(1 << (flags & 0x03));
                const uint8_t* s = c.need(size_t(nlen));
                if (std::string(reinterpret_cast<const char*>(s), size_t(nlen)) != name) continue;
                if (ltype != 0) throw FormatError("HDF5 soft or external link '" + name + "' is not supported");
                out = offset(c.need(size_t(so_)));
                return true;
            }
        }
        if (!is_group) throw FormatError("HDF5 path component before '" + name + "' is not a group");
        return false;
    }

    std::vector<uint8_t> local_heap(uint64_t addr) {
        const std::vector<uint8_t> h = bytes(addr, 8 + 2 * size_t(sl_) + size_t(so_));
        if (std::memcmp(h.data(), "HEAP", 4) != 0 || h[4] != 0) throw FormatError("HDF5 local heap");
        const uint64_t size = length(&h[8]);
        const uint64_t data = offset(&h[8 + 2 * size_t(sl_)]);
        return bytes(data, size);
    }

    bool symbol_lookup(uint64_t node, const std::vector<uint8_t>& names, const std::string& name, uint64_t& out,
                       int depth) {
        if (depth > 32) throw FormatError("HDF5 group B-tree too deep");
        const size_t head = 8 + 2 * size_t(so_);
        const std::vector<uint8_t> h = bytes(node, head);
        if (std::memcmp(h.data(), "TREE", 4) != 0 || h[4] != 0) throw FormatError("HDF5 group B-tree node");
        const int level = h[5];
        const size_t entries = size_t(le(&h[6], 2));
        const size_t stride = size_t(sl_) + size_t(so_);
        const std::vector<uint8_t> b = bytes(node + head, entries * stride + size_t(sl_));
        for (size_t e = 0; e < entries; ++e) {
            const uint64_t child_addr = offset(&b[e * stride + size_t(sl_)]);
            if (level > 0) {
                if (symbol_lookup(child_addr, names, name, out, depth + 1)) return true;
                continue;
            }
            const std::vector<uint8_t> s = bytes(child_addr, 8);
            if (std::memcmp(s.data(), "SNOD", 4) != 0 || s[4] != 1) throw FormatError("HDF5 symbol table node");
            const size_t nsym = size_t(le(&s[6], 2));
            const size_t esz = 2 * size_t(so_) + 24;
            const std::vector<uint8_t> sym = bytes(child_addr + 8, nsym * esz);
            for (size_t k = 0; k < nsym; ++k) {
                const uint64_t noff = le(&sym[k * esz], so_);
                if (noff >= names.size()) throw FormatError("HDF5 symbol name outside the local heap");
                const char* nm = reinterpret_cast<const char*>(names.data() + noff);
                const size_t nmax = names.size() - size_t(noff);
                if (strnlen(nm, nmax) == nmax) throw FormatError("HDF5 unterminated symbol name");
                if (name == nm) {
                    out = offset(&sym[k * esz + size_t(so_)]);
                    return true;
                }
            }
        }
        return false;
    }

    // -- attributes ----------------------------------------------------------
    // Attribute messages versions 1-3; dense attribute storage (an
    // Attribute Info message with a fractal heap) is refused.
    bool find_attr(const std::string& path, const std::string& name, AttrValue& out, bool decode) {
        uint64_t addr = 0;
        if (!resolve(path, addr)) throw FormatError("HDF5 object not found: " + path);
        const std::vector<Msg> msgs = header(addr);
        for (const Msg& m : msgs) {
            if (m.type == 0x15) {
                Cursor c{m.data, 0};
                c.u(1);
                const int flags = int(c.u(1));
                if (flags & 0x01) c.need(2);
                if (offset(c.need(size_t(so_))) != kUndef)
                    throw FormatError("HDF5 dense attribute storage (fractal heap) is not supported");
            }
            if (m.type != 0x0C) continue;
            Cursor c{m.data, 0};
            const int version = int(c.u(1));
            const int flags = int(c.u(1));
            const size_t nsz = size_t(c.u(2)), tsz = size_t(c.u(2)), ssz = size_t(c.u(2));
            if (version < 1 || version > 3) throw FormatError("HDF5 attribute message version");
            if (version >= 2 && (flags & 0x03)) throw FormatError("HDF5 shared attribute types are not supported");
            if (version == 3) c.u(1);  // name character set
            auto pad = [version](size_t n) { return version == 1 ? (n + 7) / 8 * 8 : n; };
            const uint8_t* nm = c.need(pad(nsz));
            std::string aname(reinterpret_cast<const char*>(nm), nsz);
            while (!aname.empty() && aname.back() == '\0') aname.pop_back();
            if (aname != name) continue;
            if (!decode) return true;
            const uint8_t* tp = c.need(pad(tsz));
            const uint8_t* sp = c.need(pad(ssz));
            const std::vector<uint8_t> tb(tp, tp + tsz), sb(sp, sp + ssz);
            datatype(tb, out.type);
            DatasetInfo space;
            dataspace(sb, space);
            out.dims = space.dims;
            out.raw.assign(m.data.begin() + long(c.p), m.data.end());
            const uint64_t n = out.count();
            if (out.type.type == ElemType::String) {
                if (n != 1) throw FormatError("HDF5 string attribute arrays are not supported");
                const size_t len = std::min(out.raw.size(), out.type.elem);
                out.text.assign(reinterpret_cast<const char*>(out.raw.data()), strnlen(
                    reinterpret_cast<const char*>(out.raw.data()), len));
            } else if (out.type.type == ElemType::VarString) {
                if (n != 1) throw FormatError("HDF5 string attribute arrays are not supported");
                if (out.raw.size() < 4 + size_t(so_) + 4) throw FormatError("HDF5 variable-length string truncated");
                const uint64_t len = le(out.raw.data(), 4);
                const uint64_t heap = offset(out.raw.data() + 4);
                const uint64_t index = le(out.raw.data() + 4 + so_, 4);
                out.text = global_heap_object(heap, index, len);
            }
            return true;
        }
        return false;
    }

    // One object of a global heap collection ("GCOL"), its first `len` bytes.
    std::string global_heap_object(uint64_t addr, uint64_t index, uint64_t len) {
        const std::vector<uint8_t> h = bytes(addr, 8 + size_t(sl_));
        if (std::memcmp(h.data(), "GCOL", 4) != 0 || h[4] != 1) throw FormatError("HDF5 global heap collection");
        const uint64_t size = length(&h[8]);
        const std::vector<uint8_t> b = bytes(addr, size);
        size_t p = 8 + size_t(sl_);
        while (p + 8 + size_t(sl_) <= b.size()) {
            const uint64_t idx = le(&b[p], 2);
            const uint64_t osz = length(&b[p + 8]);
            const size_t data = p + 8 + size_t(sl_);
            if (idx == 0) break;  // free space: the rest of the collection
            if (data + osz > b.size()) throw FormatError("HDF5 global heap object overruns its collection");
            if (idx == index) {
                if (len > osz) throw FormatError("HDF5 variable-length string longer than its heap object");
                return std::string(reinterpret_cast<const char*>(&b[data]), size_t(len));
            }
            p = data + size_t((osz + 7) / 8 * 8);
        }
        throw FormatError("HDF5 global heap object not found");
    }

    // -- datasets ------------------------------------------------------------
    DatasetInfo dataset_info(uint64_t addr, const std::string& path) {
        const std::vector<Msg> msgs = header(addr);
        DatasetInfo d;
        bool space = false, dtype = false;
        for (const Msg& m : msgs) {
            if (m.type == 0x01) {
                refuse_shared(m);
                dataspace(m.data, d);
                space = true;
            } else if (m.type == 0x03) {
                refuse_shared(m);
                datatype(m.data, d);
                dtype = true;
            } else if (m.type == 0x08) {
                layout(m.data, d);
            } else if (m.type == 0x0B) {
                refuse_shared(m);
                filters(m.data, d);
            }
        }
        if (!space || !dtype || d.layout < 0) throw FormatError("HDF5 object " + path + " is not a dataset");
        return d;
    }

    void dataspace(const std::vector<uint8_t>& b, DatasetInfo& d) {
        Cursor c{b, 0};
        const int version = int(c.u(1));
        const int rank = int(c.u(1));
        const int flags = int(c.u(1));
        if (version == 1) {
            c.need(5);
        } else if (version == 2) {
            const int kind = int(c.u(1));
            if (kind == 2) throw FormatError("HDF5 null dataspace");
        } else {
            throw FormatError("HDF5 dataspace version " + std::to_string(version));
        }
        d.dims.clear();
        for (int i = 0; i < rank; ++i) d.dims.push_back(length(c.need(size_t(sl_))));
        (void)flags;
    }

    static void datatype(const std::vector<uint8_t>& b, DatasetInfo& d) {
        Cursor c{b, 0};
        const int cv = int(c.u(1));
        const int cls = cv & 0x0F;
        const int bits0 = int(c.u(1));
        c.need(2);
        d.elem = size_t(c.u(4));
        if (cls == 0) {
            if (bits0 & 0x01) throw FormatError("HDF5 big-endian integers are not supported");
            if (d.elem != 1 && d.elem != 2 && d.elem != 4 && d.elem != 8) throw FormatError("HDF5 integer size");
            const uint64_t off = c.u(2), prec = c.u(2);
            if (off != 0 || prec != 8 * d.elem) throw FormatError("HDF5 padded integers are not supported");
            d.type = (bits0 & 0x08) ? ElemType::Int : ElemType::UInt;
        } else if (cls == 1) {
            if ((bits0 & 0x01) || (bits0 & 0x40)) throw FormatError("HDF5 non little-endian floats are not supported");
            const uint64_t off = c.u(2), prec = c.u(2);
            const uint64_t eloc = c.u(1), esize = c.u(1), mloc = c.u(1), msize = c.u(1);
            const uint64_t bias = c.u(4);
            const bool f64 = d.elem == 8 && off == 0 && prec == 64 && eloc == 52 && esize == 11 && mloc == 0 &&
                             msize == 52 && bias == 1023;
            const bool f32 = d.elem == 4 && off == 0 && prec == 32 && eloc == 23 && esize == 8 && mloc == 0 &&
                             msize == 23 && bias == 127;
            if (!f64 && !f32) throw FormatError("HDF5 non-IEEE floating-point type");
            d.type = ElemType::Float;
        } else if (cls == 3) {
            d.type = ElemType::String;
        } else if (cls == 9) {
            // variable-length: bits 0-3 of the class bits are 1 for a string
            d.type = (bits0 & 0x0F) == 1 ? ElemType::VarString : ElemType::Other;
        } else {
            d.type = ElemType::Other;
        }
    }

    void layout(const std::vector<uint8_t>& b, DatasetInfo& d) {
        Cursor c{b, 0};
        const int version = int(c.u(1));
        if (version == 1 || version == 2) {
            const int ndim = int(c.u(1));
            const int cls = int(c.u(1));
            c.need(5);
            if (cls != 0) d.addr = offset(c.need(size_t(so_)));
            std::vector<uint64_t> dims;
            for (int i = 0; i < ndim; ++i) dims.push_back(c.u(4));
            d.layout = cls;
            if (cls == 0) {
                const uint64_t n = c.u(4);
                const uint8_t* p = c.need(size_t(n));
                d.compact.assign(p, p + n);
            } else if (cls == 2) {
                if (dims.empty()) throw FormatError("HDF5 chunked layout without dimensions");
                d.chunk.assign(dims.begin(), dims.end() - 1);
            }
            return;
        }
        if (version != 3 && version != 4) throw FormatError("HDF5 data layout version " + std::to_string(version));
        const int cls = int(c.u(1));
        d.layout = cls;
        if (cls == 0) {
            const uint64_t n = c.u(2);
            const uint8_t* p = c.need(size_t(n));
            d.compact.assign(p, p + n);
        } else if (cls == 1) {
            d.addr = offset(c.need(size_t(so_)));
            d.size = length(c.need(size_t(sl_)));
        } else if (cls == 2 && version == 3) {
            const int ndim = int(c.u(1));
            d.addr = offset(c.need(size_t(so_)));
            std::vector<uint64_t> dims;
            for (int i = 0; i < ndim; ++i) dims.push_back(c.u(4));
            if (dims.empty()) throw FormatError("HDF5 chunked layout without dimensions");
            d.chunk.assign(dims.begin(), dims.end() - 1);
            d.chunk_index = 0;
        } else if (cls == 2) {
            const int flags = int(c.u(1));
            const int ndim = int(c.u(1));
            const int enc = int(c.u(1));
            std::vector<uint64_t> dims;
            for (int i = 0; i < ndim; ++i) dims.push_back(c.u(enc));
            if (dims.empty()) throw FormatError("HDF5 chunked layout without dimensions");
            d.chunk.assign(dims.begin(), dims.end() - 1);
            const int index = int(c.u(1));
            if (index == 1) {
                if (flags & 0x02) {
                    d.single_size = length(c.need(size_t(sl_)));
                    d.single_mask = uint32_t(c.u(4));
                }
                d.addr = offset(c.need(size_t(so_)));
                d.chunk_index = 1;
            } else if (index == 2) {
                d.addr = offset(c.need(size_t(so_)));
                d.chunk_index = 2;
            } else {
                throw FormatError("HDF5 chunk index type " + std::to_string(index) +
                                  " (fixed/extensible array, version-2 B-tree) is not supported");
            }
        } else {
            throw FormatError("HDF5 virtual datasets are not supported");
        }
    }

    static void filters(const std::vector<uint8_t>& b, DatasetInfo& d) {
        Cursor c{b, 0};
        const int version = int(c.u(1));
        const int n = int(c.u(1));
        if (version == 1) c.need(6);
        else if (version != 2) throw FormatError("HDF5 filter pipeline version");
        for (int i = 0; i < n; ++i) {
            DatasetInfo::Filter f;
            f.id = uint16_t(c.u(2));
            uint64_t name_len = 0;
            if (version == 1 || f.id >= 256) name_len = c.u(2);
            c.u(2);  // flags
            const int ncv = int(c.u(2));
            if (version == 1) c.need(size_t((name_len + 7) / 8 * 8));
            else c.need(size_t(name_len));
            for (int k = 0; k < ncv; ++k) f.values.push_back(uint32_t(c.u(4)));
            if (version == 1 && (ncv & 1)) c.need(4);
            if (f.id != 1 && f.id != 2)
                throw FormatError("HDF5 filter " + std::to_string(f.id) +
                                  " is not supported (deflate and shuffle are)");
            d.filters.push_back(std::move(f));
        }
    }

    // the filters undone, last first, unless the chunk's mask skipped them
    std::vector<uint8_t> unfilter(std::vector<uint8_t> data, uint32_t mask, const DatasetInfo& d,
                                  uint64_t expect) {
        for (int i = int(d.filters.size()) - 1; i >= 0; --i) {
            if (mask & (1u << i)) continue;
            const DatasetInfo::Filter& f = d.filters[size_t(i)];
            if (f.id == 1) {
                std::vector<uint8_t> out(static_cast<size_t>(expect));
                z_stream z{};
                if (inflateInit(&z) != Z_OK) throw FormatError("zlib initialisation failed");
                z.next_in = data.data();
                z.avail_in = uInt(data.size());
                z.next_out = out.data();
                z.avail_out = uInt(out.size());
                const int rc = inflate(&z, Z_FINISH);
                const uint64_t got = z.total_out;
                inflateEnd(&z);
                if (rc != Z_STREAM_END || got != expect) throw FormatError("HDF5 deflate chunk is corrupt");
                data.swap(out);
            } else if (f.id == 2) {
                const size_t s = d.elem;
                if (s > 1) {
                    std::vector<uint8_t> out(data.size());
                    const size_t n = data.size() / s;
                    for (size_t bi = 0; bi < s; ++bi)
                        for (size_t e = 0; e < n; ++e) out[e * s + bi] = data[bi * n + e];
                    std::copy(data.begin() + long(n * s), data.end(), out.begin() + long(n * s));
                    data.swap(out);
                }
            }
        }
        if (data.size() != expect) throw FormatError("HDF5 chunk size does not match its dimensions");
        return data;
    }

    std::vector<uint8_t> raw_data(const DatasetInfo& d, const std::string& path) {
        const uint64_t n = d.count();
        if (d.elem == 0 || n > (uint64_t(1) << 62) / d.elem) throw FormatError("HDF5 dataset " + path + " size");
        const uint64_t total = n * d.elem;
        if (d.layout == 0) {
            if (d.compact.size() < total) throw FormatError("HDF5 compact dataset " + path + " truncated");
            return std::vector<uint8_t>(d.compact.begin(), d.compact.begin() + long(total));
        }
        if (d.layout == 1) {
            if (d.addr == kUndef) return std::vector<uint8_t>(size_t(total), 0);  // never written: fill 0
            if (d.size != 0 && d.size < total) throw FormatError("HDF5 dataset " + path + " extent");
            return bytes(d.addr, total);
        }
        if (d.layout != 2) throw FormatError("HDF5 data layout class " + std::to_string(d.layout));
        if (d.chunk.size() != d.dims.size()) throw FormatError("HDF5 chunk rank differs from dataset " + path);
        std::vector<uint8_t> out(static_cast<size_t>(total), 0);
        uint64_t chunk_elems = 1;
        for (uint64_t c : d.chunk) {
            if (c == 0) throw FormatError("HDF5 zero chunk dimension");
            chunk_elems *= c;
        }
        const uint64_t chunk_bytes = chunk_elems * d.elem;
        auto place = [&](const std::vector<uint64_t>& origin, const std::vector<uint8_t>& chunk) {
            scatter(d, origin, chunk, out);
        };
        if (d.addr == kUndef) return out;
        if (d.chunk_index == 0) {
            chunk_tree(d.addr, d, chunk_bytes, place, 0);
        } else {
            // single chunk / implicit index: chunks stored in row-major chunk order
            std::vector<uint64_t> nch(d.dims.size());
            uint64_t count = 1;
            for (size_t i = 0; i < d.dims.size(); ++i) {
                nch[i] = (d.dims[i] + d.chunk[i] - 1) / d.chunk[i];
                count *= nch[i];
            }
            if (d.chunk_index == 1 && count != 1) throw FormatError("HDF5 single-chunk index with several chunks");
            for (uint64_t ci = 0; ci < count; ++ci) {
                std::vector<uint64_t> origin(d.dims.size());
                uint64_t r = ci;
                for (int i = int(d.dims.size()) - 1; i >= 0; --i) {
                    origin[size_t(i)] = (r % nch[size_t(i)]) * d.chunk[size_t(i)];
                    r /= nch[size_t(i)];
                }
                const uint64_t stored = (d.chunk_index == 1 && d.single_size) ? d.single_size : chunk_bytes;
                std::vector<uint8_t> raw = bytes(d.addr + ci * chunk_bytes, stored);
                place(origin, unfilter(std::move(raw), d.single_mask, d, chunk_bytes));
            }
        }
        return out;
    }

    void chunk_tree(uint64_t node, const DatasetInfo& d, uint64_t chunk_bytes,
                    const std::function<void(const std::vector<uint64_t>&, const std::vector<uint8_t>&)>& place,
                    int depth) {
        if (depth > 32) throw FormatError("HDF5 chunk B-tree too deep");
        const size_t head = 8 + 2 * size_t(so_);
        const std::vector<uint8_t> h = bytes(node, head);
        if (std::memcmp(h.data(), "TREE", 4) != 0 || h[4] != 1) throw FormatError("HDF5 chunk B-tree node");
        const int level = h[5];
        const size_t entries = size_t(le(&h[6], 2));
        const size_t rank1 = d.dims.size() + 1;
        const size_t key = 8 + 8 * rank1;
        const size_t stride = key + size_t(so_);
        const std::vector<uint8_t> b = bytes(node + head, entries * stride + key);
        for (size_t e = 0; e < entries; ++e) {
            const uint8_t* k = &b[e * stride];
            const uint64_t child_addr = offset(k + key);
            if (level > 0) {
                chunk_tree(child_addr, d, chunk_bytes, place, depth + 1);
                continue;
            }
            const uint64_t stored = le(k, 4);
            const uint32_t mask = uint32_t(le(k + 4, 4));
            std::vector<uint64_t> origin(d.dims.size());
            for (size_t i = 0; i < d.dims.size(); ++i) origin[i] = le(k + 8 + 8 * i, 8);
            place(origin, unfilter(bytes(child_addr, stored), mask, d, chunk_bytes));
        }
    }

    static void scatter(const DatasetInfo& d, const std::vector<uint64_t>& origin, const std::vector<uint8_t>& chunk,
                        std::vector<uint8_t>& out) {
        const size_t rank = d.dims.size();
        for (size_t i = 0; i < rank; ++i)
            if (origin[i] % d.chunk[i] != 0 || origin[i] >= d.dims[i])
                throw FormatError("HDF5 chunk offset outside the dataset");
        if (rank == 0) {
            std::copy(chunk.begin(), chunk.begin() + long(d.elem), out.begin());
            return;
        }
        // copy rows along the last dimension
        const uint64_t last = std::min(d.chunk[rank - 1], d.dims[rank - 1] - origin[rank - 1]);
        std::vector<uint64_t> idx(rank, 0);
        for (;;) {
            uint64_t src = 0, dst = 0;
            bool inside = true;
            for (size_t i = 0; i < rank; ++i) {
                const uint64_t g = origin[i] + idx[i];
                if (g >= d.dims[i]) inside = false;
                src = src * d.chunk[i] + idx[i];
                dst = dst * d.dims[i] + g;
            }
            if (inside)
                std::memcpy(out.data() + dst * d.elem, chunk.data() + src * d.elem, size_t(last * d.elem));
            // advance over all but the last dimension
            int i = int(rank) - 2;
            for (; i >= 0; --i) {
                if (++idx[size_t(i)] < d.chunk[size_t(i)]) break;
                idx[size_t(i)] = 0;
            }
            if (i < 0) break;
        }
    }

    template <class T>
    static T convert(const uint8_t* p, const DatasetInfo& d) {
        if (d.type == ElemType::Float) {
            if (d.elem == 8) {
                double v;
                std::memcpy(&v, p, 8);
                return static_cast<T>(v);
            }
            float v;
            std::memcpy(&v, p, 4);
            return static_cast<T>(v);
        }
        const uint64_t u = le(p, int(d.elem));
        if (d.type == ElemType::Int) {
            const int bits = int(8 * d.elem);
            const int64_t s = bits == 64 ? int64_t(u) : (int64_t(u << (64 - bits)) >> (64 - bits));
            return static_cast<T>(s);
        }
        return static_cast<T>(u);
    }
};

}  // namespace kph5
