// HDF5 subset writer and reader for DRAGONHOARD files (host code only).
//
// On-disk structures follow the HDF5 File Format Specification 3.0:
//   superblock version 0 (II.A), version-1 object headers (IV.A.1.a) holding
//   dataspace v1, datatype v1, fill value v2, data layout v3, filter pipeline
//   v1 and attribute v1 messages (IV.A.2), symbol-table groups: local heap
//   (III.D), version-1 B-tree of type 0 (III.A.1) over symbol table nodes
//   (III.B); chunked data: version-1 B-tree of type 1 whose keys carry each
//   chunk's filtered size, filter mask and element offsets. Node sizes use the
//   format's defaults for superblock version 0: group leaf K 4, group
//   internal K 16, chunk K 32; every B-tree and symbol table node is written
//   at its full allocated size.
#include "hoard_file.h"

#include <zlib.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <set>
#include <thread>

namespace hoard {
namespace {

constexpr uint64_t kUndef = ~0ull;
constexpr int kGroupLeafK = 4, kGroupNodeK = 16, kChunkK = 32;
constexpr uint64_t kHeapFreeNull = 1;  // end of a local heap's free list

using Bytes = std::vector<uint8_t>;

void put(Bytes& v, uint64_t x, int n) {
    for (int i = 0; i < n; i++) v.push_back(uint8_t(x >> (8 * i)));
}
void put_at(Bytes& v, size_t at, uint64_t x, int n) {
    for (int i = 0; i < n; i++) v[at + i] = uint8_t(x >> (8 * i));
}
void pad8(Bytes& v) {
    while (v.size() % 8) v.push_back(0);
}
uint64_t up8(uint64_t x) { return (x + 7) & ~7ull; }
int esize_of(int type) { return type == kF64 ? 8 : 4; }

// Datatype message body, unpadded (IV.A.2.d): IEEE little-endian float of 4
// or 8 bytes, or a signed little-endian 32-bit integer.
Bytes datatype(int type) {
    Bytes v;
    if (type == kI32) {
        v.push_back(0x10);  // version 1, class 0 (fixed point)
        v.push_back(0x08);  // little-endian, zero padding, signed
        v.push_back(0);
        v.push_back(0);
        put(v, 4, 4);
        put(v, 0, 2);   // bit offset
        put(v, 32, 2);  // precision
        return v;
    }
    const bool dbl = type == kF64;
    v.push_back(0x11);  // version 1, class 1 (floating point)
    v.push_back(0x20);  // little-endian, zero padding, implied leading mantissa bit
    v.push_back(dbl ? 63 : 31);  // sign bit position
    v.push_back(0);
    put(v, dbl ? 8 : 4, 4);
    put(v, 0, 2);                 // bit offset
    put(v, dbl ? 64 : 32, 2);     // precision
    v.push_back(dbl ? 52 : 23);   // exponent location
    v.push_back(dbl ? 11 : 8);    // exponent size
    v.push_back(0);               // mantissa location
    v.push_back(dbl ? 52 : 23);   // mantissa size
    put(v, dbl ? 1023 : 127, 4);  // exponent bias
    return v;
}

// Dataspace message version 1 (IV.A.2.b); rank 0 is a scalar.
Bytes dataspace(int rank, const uint64_t* dims) {
    Bytes v;
    v.push_back(1);
    v.push_back(uint8_t(rank));
    v.push_back(0);  // no maximum dimensions
    put(v, 0, 5);
    for (int r = 0; r < rank; r++) put(v, dims[r], 8);
    return v;
}

struct Message {
    int type;
    int flags;
    Bytes body;
};

// Version-1 object header with one chunk holding every message, each padded
// to 8 bytes.
Bytes object_header(const std::vector<Message>& msgs) {
    uint64_t size = 0;
    for (const auto& m : msgs) size += 8 + up8(m.body.size());
    Bytes v;
    v.push_back(1);
    v.push_back(0);
    put(v, msgs.size(), 2);
    put(v, 1, 4);  // reference count
    put(v, size, 4);
    put(v, 0, 4);  // alignment of the first message
    for (const auto& m : msgs) {
        put(v, m.type, 2);
        put(v, up8(m.body.size()), 2);
        v.push_back(uint8_t(m.flags));
        put(v, 0, 3);
        v.insert(v.end(), m.body.begin(), m.body.end());
        pad8(v);
    }
    return v;
}

Bytes attribute(const Attr& a) {
    Bytes dt = datatype(a.type), ds = dataspace(0, nullptr);
    Bytes v;
    v.push_back(1);
    v.push_back(0);
    put(v, a.name.size() + 1, 2);
    put(v, dt.size(), 2);
    put(v, ds.size(), 2);
    v.insert(v.end(), a.name.begin(), a.name.end());
    v.push_back(0);
    pad8(v);
    v.insert(v.end(), dt.begin(), dt.end());
    pad8(v);
    v.insert(v.end(), ds.begin(), ds.end());
    pad8(v);
    if (a.type == kI32) {
        put(v, uint32_t(a.i), 4);
    } else {
        uint64_t bits;
        std::memcpy(&bits, &a.d, 8);
        put(v, bits, 8);
    }
    return v;
}

struct GroupNode {
    std::string path;
    std::map<std::string, int> children;  // name -> object id (sorted by byte order)
    uint64_t ohdr = 0, heap = 0, btree = 0;
    std::vector<uint64_t> snods;
    Bytes header;
    uint64_t heap_size = 0;
    std::vector<uint64_t> name_off;  // per child, in `children` order
};

struct DsetNode {
    const Dataset* d;
    int chunked = 0;
    uint32_t cdims[3] = {1, 1, 1};
    uint64_t nchunks = 0;
    std::vector<std::array<uint64_t, 3>> coffs;  // chunk origins, row-major order
    std::vector<Bytes> zchunks;
    uint64_t ohdr = 0, data = 0;
    std::vector<uint64_t> chunk_addr;
    // chunk B-tree: nodes per level (level 0 first), each the range of its
    // children at the level below
    std::vector<std::vector<std::pair<uint64_t, uint64_t>>> levels;
    std::vector<std::vector<uint64_t>> node_addr;
    Bytes header;
};

uint64_t group_btree_size() { return 24 + 2 * kGroupNodeK * 8 + (2 * kGroupNodeK + 1) * 8; }
uint64_t snod_size() { return 8 + 2 * kGroupLeafK * 40; }
uint64_t chunk_key_size(int rank) { return 8 + 8 * (rank + 1); }
uint64_t chunk_node_size(int rank) { return 24 + 2 * kChunkK * 8 + (2 * kChunkK + 1) * chunk_key_size(rank); }

// Chunk origins of a chunked dataset, in row-major order of the chunk grid.
void plan_chunks(DsetNode& n) {
    const Dataset& d = *n.d;
    const int r = d.rank;
    uint64_t cnt[3] = {1, 1, 1};
    for (int a = 0; a < r; a++) cnt[a] = (d.dims[a] + n.cdims[a] - 1) / n.cdims[a];
    n.nchunks = cnt[0] * cnt[1] * cnt[2];
    n.coffs.resize(n.nchunks);
    n.zchunks.assign(n.nchunks, Bytes());
    for (uint64_t c = 0; c < n.nchunks; c++) {
        uint64_t rem = c;
        std::array<uint64_t, 3> o{0, 0, 0};
        for (int a = r - 1; a >= 0; a--) {
            o[a] = (rem % cnt[a]) * n.cdims[a];
            rem /= cnt[a];
        }
        n.coffs[c] = o;
    }
}

// Gathers chunk c of n (zero past the dataset's edge) into raw and deflates
// it; false when zlib fails.
bool compress_one(DsetNode& n, uint64_t c, int level, Bytes& raw) {
    const Dataset& d = *n.d;
    const int es = esize_of(d.type);
    const int r = d.rank;
    const uint64_t C1 = r > 1 ? n.cdims[1] : 1, C2 = r > 2 ? n.cdims[2] : 1;
    raw.assign(uint64_t(n.cdims[0]) * C1 * C2 * es, 0);
    const auto& o = n.coffs[c];
    // copy the chunk's rows (the last dimension is contiguous)
    const uint64_t D1 = r > 1 ? d.dims[1] : 1, D2 = r > 2 ? d.dims[2] : 1;
    const uint64_t row = std::min<uint64_t>(n.cdims[r - 1], d.dims[r - 1] - o[r - 1]) * es;
    const uint64_t e0 = std::min<uint64_t>(n.cdims[0], d.dims[0] - o[0]);
    const uint64_t e1 = r > 1 ? std::min<uint64_t>(C1, D1 - o[1]) : 1;
    const auto* src = static_cast<const uint8_t*>(d.data);
    if (r == 1) {
        std::memcpy(raw.data(), src + o[0] * es, row);
    } else if (r == 2) {
        for (uint64_t a = 0; a < e0; a++)
            std::memcpy(raw.data() + a * C1 * es, src + ((o[0] + a) * D1 + o[1]) * es, row);
    } else {
        for (uint64_t a = 0; a < e0; a++)
            for (uint64_t b = 0; b < e1; b++)
                std::memcpy(raw.data() + (a * C1 + b) * C2 * es, src + (((o[0] + a) * D1 + o[1] + b) * D2 + o[2]) * es,
                            row);
    }
    uLongf zn = compressBound(raw.size());
    Bytes z(zn);
    if (compress2(z.data(), &zn, raw.data(), raw.size(), level) != Z_OK) return false;
    z.resize(zn);
    n.zchunks[c] = std::move(z);
    return true;
}

// Deflates every chunk of every chunked dataset: `threads` host threads take
// chunks from one shared list, so datasets do not wait for one another.
// False when any chunk failed.
bool compress_all(std::vector<DsetNode>& dn, int level, int threads) {
    std::vector<std::pair<uint32_t, uint64_t>> work;
    for (uint32_t i = 0; i < dn.size(); i++) {
        if (!dn[i].chunked) continue;
        plan_chunks(dn[i]);
        for (uint64_t c = 0; c < dn[i].nchunks; c++) work.push_back({i, c});
    }
    std::atomic<uint64_t> next{0};
    std::atomic<bool> ok{true};
    auto run = [&]() {
        Bytes raw;
        for (;;) {
            const uint64_t k = next.fetch_add(1);
            if (k >= work.size()) break;
            if (!compress_one(dn[work[k].first], work[k].second, level, raw)) ok = false;
        }
    };
    const int nt = std::max(1, std::min<int>(threads, int(std::min<uint64_t>(work.size(), 1024))));
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; t++) pool.emplace_back(run);
    run();
    for (auto& t : pool) t.join();
    return ok;
}

// Key of chunk c: filtered size, filter mask, element offsets (+ a trailing 0).
void chunk_key(Bytes& v, const DsetNode& n, uint64_t size, const std::array<uint64_t, 3>& off) {
    put(v, size, 4);
    put(v, 0, 4);
    for (int a = 0; a < n.d->rank; a++) put(v, off[a], 8);
    put(v, 0, 8);
}

std::array<uint64_t, 3> after_last(const DsetNode& n) {
    std::array<uint64_t, 3> o = n.coffs.back();
    for (int a = 0; a < n.d->rank; a++) o[a] += n.cdims[a];
    return o;
}

}  // namespace

int write_file(const std::string& path, const std::vector<Attr>& attrs, const std::vector<Dataset>& dsets, int level,
               int threads, std::string* err) {
    if (threads <= 0) threads = std::max(1u, std::thread::hardware_concurrency());
    // -- the object tree: groups (id < 0 in `children`: ~group index) and datasets
    std::vector<GroupNode> groups(1);
    groups[0].path = "/";
    std::map<std::string, int> gindex{{"/", 0}};
    std::vector<DsetNode> dn(dsets.size());
    for (size_t i = 0; i < dsets.size(); i++) {
        const std::string& p = dsets[i].path;
        if (p.empty() || p[0] != '/' || p.back() == '/') {
            *err = "dataset path must be absolute: " + p;
            return -1;
        }
        if (dsets[i].rank < 1 || dsets[i].rank > 3) {
            *err = "dataset rank must be 1 to 3: " + p;
            return -1;
        }
        int parent = 0;
        size_t at = 1;
        for (;;) {
            const size_t slash = p.find('/', at);
            const std::string name = p.substr(at, slash == std::string::npos ? std::string::npos : slash - at);
            if (name.empty()) {
                *err = "empty path component: " + p;
                return -1;
            }
            if (slash == std::string::npos) {
                if (groups[parent].children.count(name)) {
                    *err = "duplicate object: " + p;
                    return -1;
                }
                groups[parent].children[name] = int(i);
                break;
            }
            const std::string gp = p.substr(0, slash);
            auto it = gindex.find(gp);
            int g;
            if (it == gindex.end()) {
                if (groups[parent].children.count(name)) {
                    *err = "a dataset and a group share a path: " + gp;
                    return -1;
                }
                g = int(groups.size());
                groups.push_back(GroupNode{});
                groups.back().path = gp;
                gindex[gp] = g;
                groups[parent].children[name] = ~g;
            } else {
                g = it->second;
            }
            parent = g;
            at = slash + 1;
        }
        DsetNode& n = dn[i];
        n.d = &dsets[i];
        n.chunked = level > 0;
        const uint32_t cap = dsets[i].rank == 1 ? 1024 : dsets[i].rank == 2 ? 32 : 16;
        for (int a = 0; a < dsets[i].rank; a++) {
            if (dsets[i].dims[a] == 0) {
                *err = "zero-sized dataset: " + p;
                return -1;
            }
            n.cdims[a] = uint32_t(std::min<uint64_t>(dsets[i].dims[a], cap));
        }
    }
    for (auto& g : groups)
        if (g.children.size() > size_t(2 * kGroupLeafK * 2 * kGroupNodeK)) {
            *err = "too many objects in group " + g.path;
            return -1;
        }

    // -- compress every chunk
    if (!compress_all(dn, level, threads)) {
        *err = "deflate failed";
        return -1;
    }

    // -- sizes, then addresses (metadata first, raw data after)
    uint64_t at = 96;  // superblock version 0
    auto take = [&](uint64_t size) {
        const uint64_t a = at;
        at = up8(at + size);
        return a;
    };
    std::vector<Bytes> attr_bodies;
    for (const auto& a : attrs) attr_bodies.push_back(attribute(a));
    for (size_t gi = 0; gi < groups.size(); gi++) {
        GroupNode& g = groups[gi];
        std::vector<Message> msgs{{0x11, 1, Bytes(16, 0)}};
        if (gi == 0)
            for (auto& b : attr_bodies) msgs.push_back({0x0C, 0, b});
        g.header = object_header(msgs);
        g.ohdr = take(g.header.size());
        uint64_t off = 8;  // offset 0 holds the empty name
        for (const auto& c : g.children) {
            g.name_off.push_back(off);
            off += up8(c.first.size() + 1);
        }
        g.heap_size = off;
        g.heap = take(32 + g.heap_size);
        g.btree = take(group_btree_size());
        const size_t ns = (g.children.size() + 2 * kGroupLeafK - 1) / (2 * kGroupLeafK);
        for (size_t s = 0; s < std::max<size_t>(ns, 1); s++) g.snods.push_back(take(snod_size()));
    }
    for (auto& n : dn) {
        const Dataset& d = *n.d;
        std::vector<Message> msgs;
        msgs.push_back({0x01, 0, dataspace(d.rank, d.dims)});
        msgs.push_back({0x03, 1, datatype(d.type)});
        msgs.push_back({0x05, 1, Bytes{2, uint8_t(n.chunked ? 3 : 2), 2, 0}});
        Bytes layout;
        if (n.chunked) {
            layout = {3, 2, uint8_t(d.rank + 1)};
            put(layout, 0, 8);
            for (int a = 0; a < d.rank; a++) put(layout, n.cdims[a], 4);
            put(layout, esize_of(d.type), 4);
            Bytes pipe{1, 1};
            put(pipe, 0, 6);
            put(pipe, 1, 2);  // deflate
            put(pipe, 8, 2);  // name length
            put(pipe, 1, 2);  // optional filter
            put(pipe, 1, 2);  // one client value
            const char nm[8] = {'d', 'e', 'f', 'l', 'a', 't', 'e', 0};
            pipe.insert(pipe.end(), nm, nm + 8);
            put(pipe, level, 4);
            put(pipe, 0, 4);
            msgs.push_back({0x0B, 1, pipe});
        } else {
            layout = {3, 1};
            put(layout, 0, 8);
            put(layout, 0, 8);
        }
        msgs.push_back({0x08, 0, layout});
        n.header = object_header(msgs);
        n.ohdr = take(n.header.size());
        if (n.chunked) {
            // level 0 groups the chunks, each higher level groups the nodes below
            uint64_t count = n.nchunks;
            do {
                std::vector<std::pair<uint64_t, uint64_t>> lv;
                for (uint64_t s = 0; s < count; s += 2 * kChunkK) lv.push_back({s, std::min<uint64_t>(count, s + 2 * kChunkK)});
                n.levels.push_back(lv);
                std::vector<uint64_t> addr;
                for (size_t k = 0; k < lv.size(); k++) addr.push_back(take(chunk_node_size(d.rank)));
                n.node_addr.push_back(addr);
                count = lv.size();
            } while (count > 1);
        }
    }
    const uint64_t meta_end = at;
    for (auto& n : dn) {
        if (n.chunked) {
            n.chunk_addr.resize(n.nchunks);
            for (uint64_t c = 0; c < n.nchunks; c++) n.chunk_addr[c] = take(n.zchunks[c].size());
        } else {
            uint64_t bytes = esize_of(n.d->type);
            for (int a = 0; a < n.d->rank; a++) bytes *= n.d->dims[a];
            n.data = take(bytes);
        }
    }
    const uint64_t eof = at;

    // -- encode the metadata
    Bytes meta(meta_end, 0);
    auto place = [&](uint64_t addr, const Bytes& b) { std::memcpy(meta.data() + addr, b.data(), b.size()); };
    {
        Bytes sb;
        const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
        sb.insert(sb.end(), sig, sig + 8);
        sb.push_back(0);  // superblock version
        sb.push_back(0);  // free-space storage version
        sb.push_back(0);  // root group symbol table entry version
        sb.push_back(0);
        sb.push_back(0);  // shared header message format version
        sb.push_back(8);  // size of offsets
        sb.push_back(8);  // size of lengths
        sb.push_back(0);
        put(sb, kGroupLeafK, 2);
        put(sb, kGroupNodeK, 2);
        put(sb, 0, 4);  // file consistency flags
        put(sb, 0, 8);  // base address
        put(sb, kUndef, 8);
        put(sb, eof, 8);
        put(sb, kUndef, 8);
        // root group symbol table entry, with the cached B-tree and heap
        put(sb, 0, 8);
        put(sb, groups[0].ohdr, 8);
        put(sb, 1, 4);
        put(sb, 0, 4);
        put(sb, groups[0].btree, 8);
        put(sb, groups[0].heap, 8);
        place(0, sb);
    }
    for (auto& g : groups) {
        Bytes h = g.header;
        put_at(h, 16 + 8, g.btree, 8);
        put_at(h, 16 + 16, g.heap, 8);
        place(g.ohdr, h);
        Bytes hp{'H', 'E', 'A', 'P', 0, 0, 0, 0};
        put(hp, g.heap_size, 8);
        put(hp, kHeapFreeNull, 8);
        put(hp, g.heap + 32, 8);
        hp.resize(32 + g.heap_size, 0);
        size_t k = 0;
        for (const auto& c : g.children) std::memcpy(hp.data() + 32 + g.name_off[k++], c.first.data(), c.first.size());
        place(g.heap, hp);
        // symbol table nodes of up to 2 * leaf K entries, names in byte order
        std::vector<std::pair<std::string, int>> kids(g.children.begin(), g.children.end());
        const size_t per = 2 * kGroupLeafK;
        Bytes bt{'T', 'R', 'E', 'E', 0, 0};
        put(bt, g.snods.size(), 2);
        put(bt, kUndef, 8);
        put(bt, kUndef, 8);
        put(bt, 0, 8);  // key 0: the empty name
        for (size_t s = 0; s < g.snods.size(); s++) {
            const size_t lo = s * per, hi = std::min(kids.size(), lo + per);
            Bytes sn{'S', 'N', 'O', 'D', 1, 0};
            put(sn, hi - lo, 2);
            for (size_t e = lo; e < hi; e++) {
                const int id = kids[e].second;
                put(sn, g.name_off[e], 8);
                if (id < 0) {
                    const GroupNode& cg = groups[~id];
                    put(sn, cg.ohdr, 8);
                    put(sn, 1, 4);
                    put(sn, 0, 4);
                    put(sn, cg.btree, 8);
                    put(sn, cg.heap, 8);
                } else {
                    put(sn, dn[id].ohdr, 8);
                    put(sn, 0, 4);
                    put(sn, 0, 4);
                    put(sn, 0, 16);
                }
            }
            sn.resize(snod_size(), 0);
            place(g.snods[s], sn);
            put(bt, g.snods[s], 8);
            put(bt, hi > lo ? g.name_off[hi - 1] : 0, 8);  // largest name in the node
        }
        bt.resize(group_btree_size(), 0);
        place(g.btree, bt);
    }
    for (auto& n : dn) {
        Bytes h = n.header;
        // the layout message is the last one: patch its address
        const size_t lay = h.size() - up8(n.chunked ? 3 + 8 + 4 * (n.d->rank + 1) : 18);
        put_at(h, lay + (n.chunked ? 3 : 2), n.chunked ? n.node_addr.back()[0] : n.data, 8);
        if (!n.chunked) {
            uint64_t bytes = esize_of(n.d->type);
            for (int a = 0; a < n.d->rank; a++) bytes *= n.d->dims[a];
            put_at(h, lay + 10, bytes, 8);
        }
        place(n.ohdr, h);
        if (!n.chunked) continue;
        // left key of every entry at every level: the first chunk below it
        std::vector<uint64_t> first(n.levels[0].size());
        for (size_t L = 0; L < n.levels.size(); L++) {
            const auto& lv = n.levels[L];
            std::vector<uint64_t> nfirst(lv.size());
            for (size_t k = 0; k < lv.size(); k++) {
                Bytes nd{'T', 'R', 'E', 'E', 1, uint8_t(L)};
                put(nd, lv[k].second - lv[k].first, 2);
                put(nd, k > 0 ? n.node_addr[L][k - 1] : kUndef, 8);
                put(nd, k + 1 < lv.size() ? n.node_addr[L][k + 1] : kUndef, 8);
                for (uint64_t e = lv[k].first; e < lv[k].second; e++) {
                    const uint64_t c = L == 0 ? e : first[e];
                    chunk_key(nd, n, n.zchunks[c].size(), n.coffs[c]);
                    put(nd, L == 0 ? n.chunk_addr[e] : n.node_addr[L - 1][e], 8);
                }
                // right key: the next node's first chunk, or one chunk past the last
                const uint64_t nextc = L == 0 ? lv[k].second : (lv[k].second < first.size() ? first[lv[k].second] : n.nchunks);
                if (nextc < n.nchunks) chunk_key(nd, n, n.zchunks[nextc].size(), n.coffs[nextc]);
                else chunk_key(nd, n, 0, after_last(n));
                nd.resize(chunk_node_size(n.d->rank), 0);
                place(n.node_addr[L][k], nd);
                nfirst[k] = L == 0 ? lv[k].first : first[lv[k].first];
            }
            first = nfirst;
        }
    }

    // -- write
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) {
        *err = "cannot open " + path + " for writing";
        return -1;
    }
    bool ok = std::fwrite(meta.data(), 1, meta.size(), f) == meta.size();
    uint64_t pos = meta.size();
    static const uint8_t zeros[8] = {0};
    auto seek_to = [&](uint64_t a) {
        while (ok && pos < a) {
            const size_t k = size_t(std::min<uint64_t>(8, a - pos));
            ok = std::fwrite(zeros, 1, k, f) == k;
            pos += k;
        }
    };
    for (auto& n : dn) {
        if (n.chunked) {
            for (uint64_t c = 0; c < n.nchunks && ok; c++) {
                seek_to(n.chunk_addr[c]);
                ok = ok && std::fwrite(n.zchunks[c].data(), 1, n.zchunks[c].size(), f) == n.zchunks[c].size();
                pos += n.zchunks[c].size();
            }
        } else {
            uint64_t bytes = esize_of(n.d->type);
            for (int a = 0; a < n.d->rank; a++) bytes *= n.d->dims[a];
            seek_to(n.data);
            ok = ok && std::fwrite(n.d->data, 1, bytes, f) == bytes;
            pos += bytes;
        }
    }
    seek_to(eof);
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) {
        *err = "write failed: " + path;
        return -1;
    }
    return 0;
}

// ===========================================================================
// Reader
// ===========================================================================
namespace {
uint64_t get(const std::vector<uint8_t>& d, size_t at, int n) {
    uint64_t x = 0;
    for (int i = 0; i < n; i++) x |= uint64_t(d[at + i]) << (8 * i);
    return x;
}
bool fail_with(std::string* err, const std::string& m) {
    *err = m;
    return false;
}
}  // namespace

bool File::open(const std::string& path, std::string* err) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return fail_with(err, "cannot open " + path);
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    d_.resize(n > 0 ? size_t(n) : 0);
    const bool ok = n > 0 && std::fread(d_.data(), 1, d_.size(), f) == d_.size();
    std::fclose(f);
    if (!ok) return fail_with(err, "cannot read " + path);
    static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    size_t sb = std::string::npos;
    for (size_t off = 0; off + 8 <= d_.size(); off = off ? off * 2 : 512) {
        if (std::memcmp(d_.data() + off, sig, 8) == 0) {
            sb = off;
            break;
        }
    }
    if (sb == std::string::npos) return fail_with(err, path + " is not an HDF5 file");
    if (!in_file(sb, 96)) return fail_with(err, "truncated superblock");
    const int ver = d_[sb + 8];
    if (ver > 1) return fail_with(err, "HDF5 superblock version " + std::to_string(ver) + " is not supported");
    if (d_[sb + 13] != 8 || d_[sb + 14] != 8) return fail_with(err, "only 8-byte offsets and lengths are supported");
    const size_t p = sb + (ver == 0 ? 24 : 28);
    if (!in_file(p, 72)) return fail_with(err, "truncated superblock");
    const uint64_t base = get(d_, p, 8);
    base_ = base == 0 ? sb : base;
    root_ = get(d_, p + 32 + 8, 8);
    return true;
}

bool File::header(uint64_t addr, std::vector<Msg>* msgs, std::string* err) const {
    uint64_t a = base_ + addr;
    if (!in_file(a, 16)) return fail_with(err, "object header outside the file");
    if (std::memcmp(d_.data() + a, "OHDR", 4) == 0) return fail_with(err, "version-2 object headers are not supported");
    if (d_[a] != 1) return fail_with(err, "unknown object header version");
    const uint64_t nmsg = get(d_, a + 2, 2);
    std::vector<std::pair<uint64_t, uint64_t>> blocks{{a + 16, get(d_, a + 8, 4)}};
    uint64_t seen = 0;
    for (size_t b = 0; b < blocks.size() && seen < nmsg; b++) {
        const uint64_t start = blocks[b].first, len = blocks[b].second;
        if (!in_file(start, len)) return fail_with(err, "object header chunk outside the file");
        uint64_t q = start;
        while (q + 8 <= start + len && seen < nmsg) {
            const int type = int(get(d_, q, 2));
            const uint64_t size = get(d_, q + 2, 2);
            const int flags = d_[q + 4];
            if (q + 8 + size > start + len) return fail_with(err, "object header message overruns its chunk");
            if (flags & 0x02) return fail_with(err, "shared object header messages are not supported");
            if (type == 0x10) {
                if (size < 16) return fail_with(err, "bad continuation message");
                blocks.push_back({base_ + get(d_, q + 8, 8), get(d_, q + 16, 8)});
                if (blocks.size() > 4096) return fail_with(err, "too many continuation blocks");
            } else if (type != 0) {
                msgs->push_back({type, size_t(q + 8), size_t(size)});
            }
            seen++;
            q += 8 + size;
        }
    }
    return true;
}

bool File::heap(uint64_t addr, std::vector<uint8_t>* out, std::string* err) const {
    const uint64_t a = base_ + addr;
    if (!in_file(a, 32) || std::memcmp(d_.data() + a, "HEAP", 4) != 0) return fail_with(err, "bad local heap");
    const uint64_t size = get(d_, a + 8, 8), data = base_ + get(d_, a + 24, 8);
    if (!in_file(data, size)) return fail_with(err, "local heap outside the file");
    out->assign(d_.begin() + data, d_.begin() + data + size);
    return true;
}

bool File::group_btree(uint64_t addr, const std::vector<uint8_t>& names,
                       std::vector<std::pair<std::string, uint64_t>>* out, int depth, std::string* err) const {
    if (depth > 32) return fail_with(err, "group B-tree too deep");
    const uint64_t a = base_ + addr;
    if (!in_file(a, 24) || std::memcmp(d_.data() + a, "TREE", 4) != 0 || d_[a + 4] != 0)
        return fail_with(err, "bad group B-tree node");
    const int lvl = d_[a + 5];
    const uint64_t used = get(d_, a + 6, 2);
    if (!in_file(a + 24, 8 + used * 16)) return fail_with(err, "group B-tree node outside the file");
    for (uint64_t e = 0; e < used; e++) {
        const uint64_t child = get(d_, a + 24 + 8 + e * 16, 8);
        if (lvl > 0) {
            if (!group_btree(child, names, out, depth + 1, err)) return false;
            continue;
        }
        const uint64_t s = base_ + child;
        if (!in_file(s, 8) || std::memcmp(d_.data() + s, "SNOD", 4) != 0) return fail_with(err, "bad symbol table node");
        const uint64_t n = get(d_, s + 6, 2);
        if (!in_file(s + 8, n * 40)) return fail_with(err, "symbol table node outside the file");
        for (uint64_t k = 0; k < n; k++) {
            const uint64_t off = get(d_, s + 8 + 40 * k, 8);
            if (off >= names.size()) return fail_with(err, "link name outside the heap");
            const char* nm = reinterpret_cast<const char*>(names.data() + off);
            out->push_back({std::string(nm, strnlen(nm, names.size() - off)), get(d_, s + 8 + 40 * k + 8, 8)});
        }
    }
    return true;
}

bool File::links(const std::vector<Msg>& msgs, std::vector<std::pair<std::string, uint64_t>>* out,
                 std::string* err) const {
    for (const auto& m : msgs) {
        if (m.type == 0x11) {
            std::vector<uint8_t> names;
            if (!heap(get(d_, m.body + 8, 8), &names, err)) return false;
            if (!group_btree(get(d_, m.body, 8), names, out, 0, err)) return false;
        } else if (m.type == 0x06) {  // link message of a compact group (IV.A.2.g)
            size_t q = m.body + 1;
            const int flags = d_[q++];
            int ltype = 0;
            if (flags & 0x08) ltype = d_[q++];
            if (flags & 0x04) q += 8;
            if (flags & 0x10) q++;
            const int nls = 1 << (flags & 3);
            const uint64_t nlen = get(d_, q, nls);
            q += nls;
            std::string name(reinterpret_cast<const char*>(d_.data() + q), nlen);
            q += nlen;
            if (ltype == 0) out->push_back({name, get(d_, q, 8)});
        }
    }
    return true;
}

bool File::lookup(const std::string& path, uint64_t* addr, std::string* err) const {
    uint64_t cur = root_;
    size_t at = 0;
    while (at < path.size()) {
        while (at < path.size() && path[at] == '/') at++;
        if (at >= path.size()) break;
        size_t end = path.find('/', at);
        if (end == std::string::npos) end = path.size();
        const std::string name = path.substr(at, end - at);
        std::vector<Msg> msgs;
        if (!header(cur, &msgs, err)) return false;
        std::vector<std::pair<std::string, uint64_t>> ls;
        if (!links(msgs, &ls, err)) return false;
        bool found = false;
        for (auto& l : ls)
            if (l.first == name) {
                cur = l.second;
                found = true;
                break;
            }
        if (!found) return fail_with(err, "no object " + path);
        at = end;
    }
    *addr = cur;
    return true;
}

bool File::has(const std::string& path) const {
    uint64_t a;
    std::string e;
    return lookup(path, &a, &e);
}

namespace {
struct TypeInfo {
    int cls = -1, size = 0;
    bool sgn = false, be = false;
};
bool parse_type(const std::vector<uint8_t>& d, size_t b, TypeInfo* t, std::string* err) {
    t->cls = d[b] & 0x0F;
    t->be = d[b + 1] & 1;
    t->sgn = (d[b + 1] >> 3) & 1;
    t->size = int(get(d, b + 4, 4));
    if (t->cls == 1 && (t->size == 4 || t->size == 8)) return true;
    if (t->cls == 0 && (t->size == 1 || t->size == 2 || t->size == 4 || t->size == 8)) return true;
    return fail_with(err, "unsupported datatype (class " + std::to_string(t->cls) + ", " + std::to_string(t->size) + " bytes)");
}
double elem(const uint8_t* p, const TypeInfo& t) {
    uint8_t b[8];
    for (int i = 0; i < t.size; i++) b[i] = t.be ? p[t.size - 1 - i] : p[i];
    if (t.cls == 1) {
        if (t.size == 8) {
            double x;
            std::memcpy(&x, b, 8);
            return x;
        }
        float x;
        std::memcpy(&x, b, 4);
        return x;
    }
    uint64_t u = 0;
    std::memcpy(&u, b, t.size);
    if (t.sgn && t.size < 8 && (u >> (8 * t.size - 1)) & 1) u |= ~0ull << (8 * t.size);
    return t.sgn ? double(int64_t(u)) : double(u);
}
bool parse_space(const std::vector<uint8_t>& d, size_t b, std::vector<uint64_t>* dims, std::string* err) {
    const int ver = d[b], rank = d[b + 1];
    size_t q;
    if (ver == 1) q = b + 8;
    else if (ver == 2) {
        if (d[b + 3] == 0) {  // scalar
            dims->clear();
            return true;
        }
        q = b + 4;
    } else return fail_with(err, "unsupported dataspace version");
    dims->resize(rank);
    for (int r = 0; r < rank; r++) (*dims)[r] = get(d, q + 8 * r, 8);
    return true;
}
}  // namespace

bool File::attr(const std::string& name, double* value, std::string* err) const {
    std::vector<Msg> msgs;
    if (!header(root_, &msgs, err)) return false;
    for (const auto& m : msgs) {
        if (m.type != 0x0C) continue;
        const int ver = d_[m.body];
        const uint64_t nsz = get(d_, m.body + 2, 2), tsz = get(d_, m.body + 4, 2), ssz = get(d_, m.body + 6, 2);
        size_t q = m.body + 8 + (ver == 3 ? 1 : 0);
        auto adv = [&](uint64_t n) { return ver == 1 ? (n + 7) / 8 * 8 : n; };
        const std::string nm(reinterpret_cast<const char*>(d_.data() + q), strnlen(reinterpret_cast<const char*>(d_.data() + q), nsz));
        if (nm != name) continue;
        q += adv(nsz);
        TypeInfo t;
        if (!parse_type(d_, q, &t, err)) return false;
        q += adv(tsz);
        q += adv(ssz);
        if (!in_file(q, t.size)) return fail_with(err, "attribute data outside the file");
        *value = elem(d_.data() + q, t);
        return true;
    }
    return fail_with(err, "no attribute " + name);
}

bool File::shape(const std::string& path, std::vector<uint64_t>* dims, std::string* err) const {
    uint64_t a;
    if (!lookup(path, &a, err)) return false;
    std::vector<Msg> msgs;
    if (!header(a, &msgs, err)) return false;
    for (const auto& m : msgs)
        if (m.type == 0x01) return parse_space(d_, m.body, dims, err);
    return fail_with(err, path + " is not a dataset");
}

bool File::chunk_btree(uint64_t addr, int rank1, const std::vector<uint32_t>& chunk, const std::vector<uint64_t>& dims,
                       int esize, int cls, bool sgn, bool be,
                       const std::vector<std::pair<int, std::vector<uint32_t>>>& filters, std::vector<double>* out,
                       int depth, std::string* err) const {
    if (depth > 32) return fail_with(err, "chunk B-tree too deep");
    const uint64_t a = base_ + addr;
    if (!in_file(a, 24) || std::memcmp(d_.data() + a, "TREE", 4) != 0 || d_[a + 4] != 1)
        return fail_with(err, "bad chunk B-tree node");
    const int lvl = d_[a + 5];
    const uint64_t used = get(d_, a + 6, 2);
    const uint64_t ks = 8 + 8 * uint64_t(rank1);
    if (!in_file(a + 24, used * (ks + 8) + ks)) return fail_with(err, "chunk B-tree node outside the file");
    const int rank = rank1 - 1;
    uint64_t celems = 1;
    for (int r = 0; r < rank; r++) celems *= chunk[r];
    TypeInfo t;
    t.cls = cls;
    t.size = esize;
    t.sgn = sgn;
    t.be = be;
    for (uint64_t e = 0; e < used; e++) {
        const size_t k = a + 24 + e * (ks + 8);
        const uint64_t csize = get(d_, k, 4), mask = get(d_, k + 4, 4);
        std::vector<uint64_t> off(rank);
        for (int r = 0; r < rank; r++) off[r] = get(d_, k + 8 + 8 * r, 8);
        const uint64_t child = get(d_, k + ks, 8);
        if (lvl > 0) {
            if (!chunk_btree(child, rank1, chunk, dims, esize, cls, sgn, be, filters, out, depth + 1, err)) return false;
            continue;
        }
        if (!in_file(base_ + child, csize)) return fail_with(err, "chunk outside the file");
        std::vector<uint8_t> raw(d_.begin() + base_ + child, d_.begin() + base_ + child + csize);
        for (int f = int(filters.size()) - 1; f >= 0; f--) {
            if (mask & (1u << f)) continue;
            const int id = filters[f].first;
            if (id == 1) {
                std::vector<uint8_t> z(celems * esize);
                uLongf zn = z.size();
                if (uncompress(z.data(), &zn, raw.data(), raw.size()) != Z_OK) return fail_with(err, "inflate failed");
                z.resize(zn);
                raw.swap(z);
            } else if (id == 2) {
                std::vector<uint8_t> s(raw.size());
                const size_t n = raw.size() / esize;
                for (size_t i = 0; i < n; i++)
                    for (int b = 0; b < esize; b++) s[i * esize + b] = raw[b * n + i];
                raw.swap(s);
            } else if (id == 3) {
                if (raw.size() >= 4) raw.resize(raw.size() - 4);
            } else {
                return fail_with(err, "unsupported filter " + std::to_string(id));
            }
        }
        if (raw.size() < celems * esize) return fail_with(err, "short chunk");
        // scatter the chunk into the row-major output
        std::vector<uint64_t> ext(rank);
        for (int r = 0; r < rank; r++) {
            if (off[r] >= dims[r]) return fail_with(err, "chunk offset outside the dataset");
            ext[r] = std::min<uint64_t>(chunk[r], dims[r] - off[r]);
        }
        std::vector<uint64_t> idx(rank, 0);
        for (;;) {
            uint64_t src = 0, dst = 0;
            for (int r = 0; r < rank; r++) {
                src = src * chunk[r] + idx[r];
                dst = dst * dims[r] + off[r] + idx[r];
            }
            (*out)[dst] = elem(raw.data() + src * esize, t);
            int r = rank - 1;
            while (r >= 0 && ++idx[r] == ext[r]) idx[r--] = 0;
            if (r < 0) break;
        }
    }
    return true;
}

bool File::read(const std::string& path, std::vector<double>* out, std::string* err) const {
    uint64_t a;
    if (!lookup(path, &a, err)) return false;
    std::vector<Msg> msgs;
    if (!header(a, &msgs, err)) return false;
    std::vector<uint64_t> dims;
    TypeInfo t;
    size_t lay = 0;
    bool have_space = false, have_type = false;
    std::vector<std::pair<int, std::vector<uint32_t>>> filters;
    for (const auto& m : msgs) {
        if (m.type == 0x01) {
            if (!parse_space(d_, m.body, &dims, err)) return false;
            have_space = true;
        } else if (m.type == 0x03) {
            if (!parse_type(d_, m.body, &t, err)) return false;
            have_type = true;
        } else if (m.type == 0x08) {
            lay = m.body;
        } else if (m.type == 0x0B) {
            const int ver = d_[m.body], nf = d_[m.body + 1];
            size_t q = m.body + (ver == 1 ? 8 : 2);
            for (int f = 0; f < nf; f++) {
                const int id = int(get(d_, q, 2));
                uint64_t nlen = 0, ncd;
                if (ver == 1 || id >= 256) {
                    nlen = get(d_, q + 2, 2);
                    ncd = get(d_, q + 6, 2);
                    q += 8 + (ver == 1 ? (nlen + 7) / 8 * 8 : nlen);
                } else {
                    ncd = get(d_, q + 4, 2);
                    q += 6;
                }
                std::vector<uint32_t> cd(ncd);
                for (uint64_t c = 0; c < ncd; c++) cd[c] = uint32_t(get(d_, q + 4 * c, 4));
                q += 4 * ncd + ((ver == 1 && (ncd & 1)) ? 4 : 0);
                filters.push_back({id, cd});
            }
        }
    }
    if (!have_space || !have_type || !lay) return fail_with(err, path + " is not a dataset");
    uint64_t n = 1;
    for (auto x : dims) n *= x;
    out->assign(n, 0.0);
    const int ver = d_[lay];
    int cls;
    size_t q;
    if (ver == 1 || ver == 2) {
        cls = d_[lay + 2];
        q = lay + 8;
    } else if (ver == 3) {
        cls = d_[lay + 1];
        q = lay + 2;
    } else {
        return fail_with(err, "unsupported layout message version");
    }
    if (cls == 0 && ver == 3) {
        const uint64_t size = get(d_, q, 2);
        if (size < n * t.size) return fail_with(err, "short compact dataset");
        for (uint64_t i = 0; i < n; i++) (*out)[i] = elem(d_.data() + q + 2 + i * t.size, t);
        return true;
    }
    if (cls == 1) {
        const uint64_t addr = get(d_, q, 8);
        if (addr == kUndef) return true;
        if (!in_file(base_ + addr, n * t.size)) return fail_with(err, "dataset outside the file");
        for (uint64_t i = 0; i < n; i++) (*out)[i] = elem(d_.data() + base_ + addr + i * t.size, t);
        return true;
    }
    if (cls != 2) return fail_with(err, "unsupported layout class");
    int rank1;
    uint64_t bt;
    size_t cq;
    if (ver == 3) {
        rank1 = d_[q];
        bt = get(d_, q + 1, 8);
        cq = q + 9;
    } else {
        rank1 = d_[lay + 1];
        bt = get(d_, q, 8);
        cq = q + 8;
    }
    if (rank1 != int(dims.size()) + 1) return fail_with(err, "chunk rank does not match the dataspace");
    std::vector<uint32_t> chunk(rank1);
    for (int r = 0; r < rank1; r++) chunk[r] = uint32_t(get(d_, cq + 4 * r, 4));
    if (bt == kUndef) return true;
    return chunk_btree(bt, rank1, chunk, dims, t.size, t.cls, t.sgn, t.be, filters, out, 0, err);
}

}  // namespace hoard
