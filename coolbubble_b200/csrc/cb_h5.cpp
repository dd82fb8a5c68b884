/* cb_h5.cpp -- native HDF5 writer for field snapshots (no libhdf5).
 *
 * The reference writes each field snapshot through the HDF5 C++ library
 * (Bubble::OutField, src/bubble.cpp:887-953): float datasets phi, pi (and
 * Ekin, gradphi, potEnergy) of shape (n,)*D in lattice order, chunked
 * (1-D: the whole field; 2-D: min(n, max(1, 65536 / n)) rows; 3-D: one
 * plane), shuffled and deflated at level 9, and the scalar double attributes
 * D, L, nGrids, reduc, c, t, a on the root group. libhdf5 is not part of this
 * build, so the file is laid out here, in the format libhdf5 writes with its
 * default ("earliest") format bounds, which every HDF5 reader since 1.8 opens:
 *
 *   superblock version 0: offsets and lengths of 8 bytes, group leaf K 4,
 *     group internal K 16, base address 0;
 *   root group: version-1 object header holding a symbol-table message and
 *     one version-1 attribute message per attribute; a local heap with the
 *     link names; a version-1 B-tree (type 0) whose one leaf points at one
 *     symbol-table node (entries sorted by name, at most 2 * 4 of them);
 *   each dataset: version-1 object header with dataspace (version 1, maximum
 *     dimensions = dimensions), datatype (IEEE float, little endian), fill
 *     value (version 2, library default), filter pipeline (version 1:
 *     shuffle, deflate) and layout (version 3, chunked) messages; the chunk
 *     index is a version-1 B-tree (type 1) of nodes with room for 2K = 64
 *     entries (the K that readers assume for version-0 superblocks), with as
 *     many levels as the chunk count needs.
 *
 * Each chunk is gathered (an edge chunk is padded with the fill value 0, as
 * libhdf5 stores it), byte-shuffled and compressed with zlib's compress2 at
 * the given level, which is what HDF5's deflate filter does. A chunk whose
 * compressed form would exceed its raw size is stored shuffled only, with the
 * deflate bit set in its filter mask: libhdf5's outcome for an optional
 * filter that fails. Chunks are compressed in parallel on the host threads,
 * in batches, and written in chunk order, so the file's bytes do not depend
 * on the thread count.
 */
#include <zlib.h>
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "coolbubble_b200.h"
#include "cb_handle.h"

using cb::fail;

namespace {

constexpr uint64_t UNDEF = ~uint64_t(0);
constexpr int GROUP_LEAF_K = 4;        /* symbol-table node: 2K = 8 entries */
constexpr int GROUP_INTERNAL_K = 16;   /* group B-tree node: 2K = 32 children */
constexpr int CHUNK_K = 32;            /* chunk B-tree node: 2K = 64 children */
constexpr size_t SUPERBLOCK_BYTES = 96;
constexpr size_t ENTRY_BYTES = 40;     /* symbol-table entry */
constexpr int MAX_SETS = 2 * GROUP_LEAF_K;
constexpr unsigned FILTER_DEFLATE = 1, FILTER_SHUFFLE = 2;
constexpr unsigned MSG_DATASPACE = 0x1, MSG_DATATYPE = 0x3, MSG_FILL = 0x5, MSG_LAYOUT = 0x8,
                   MSG_PIPELINE = 0xB, MSG_ATTRIBUTE = 0xC, MSG_SYMBOL_TABLE = 0x11;
constexpr unsigned MSG_CONSTANT = 1;

size_t pad8(size_t x) { return (x + 7) & ~size_t(7); }

/* little-endian byte buffer */
struct Bytes {
    std::vector<uint8_t> b;
    void u8(unsigned v) { b.push_back((uint8_t)v); }
    void u16(unsigned v) { u8(v & 0xffu); u8((v >> 8) & 0xffu); }
    void u32(uint32_t v) { for (int i = 0; i < 4; ++i) u8((v >> (8 * i)) & 0xffu); }
    void u64(uint64_t v) { for (int i = 0; i < 8; ++i) u8(unsigned((v >> (8 * i)) & 0xffu)); }
    void raw(const void *p, size_t n) {
        const uint8_t *q = (const uint8_t *)p;
        b.insert(b.end(), q, q + n);
    }
    void add(const Bytes &o) { b.insert(b.end(), o.b.begin(), o.b.end()); }
    void zeros(size_t n) { b.insert(b.end(), n, 0); }
    void align8() { zeros(pad8(b.size()) - b.size()); }
    size_t size() const { return b.size(); }
};

/* datatype message body: IEEE float of 4 or 8 bytes, little endian (20 bytes) */
Bytes float_type(int bytes) {
    Bytes t;
    t.u8(0x11);                                  /* version 1, class 1 (floating point) */
    t.u8(0x20);                                  /* little endian, mantissa's leading bit implied */
    t.u8(bytes == 4 ? 31 : 63);                  /* sign bit position */
    t.u8(0);
    t.u32(bytes);
    t.u16(0);                                    /* bit offset */
    t.u16(8 * bytes);                            /* precision */
    if (bytes == 4) {
        t.u8(23); t.u8(8); t.u8(0); t.u8(23); t.u32(127);     /* exponent at 23, 8 bits; mantissa 0..22; bias */
    } else {
        t.u8(52); t.u8(11); t.u8(0); t.u8(52); t.u32(1023);
    }
    return t;
}

/* dataspace message body, version 1 (rank 0 = scalar) */
Bytes dataspace(int rank, const uint64_t *dims) {
    Bytes s;
    s.u8(1);
    s.u8(rank);
    s.u8(rank ? 1 : 0);                          /* maximum dimensions present */
    s.u8(0);
    s.u32(0);
    for (int a = 0; a < rank; ++a) s.u64(dims[a]);
    for (int a = 0; a < rank; ++a) s.u64(dims[a]);
    return s;
}

/* messages of a version-1 object header */
struct Header {
    Bytes msgs;
    int count = 0;
    void add(unsigned type, unsigned flags, const Bytes &body) {
        const size_t n = pad8(body.size());
        msgs.u16(type);
        msgs.u16((unsigned)n);
        msgs.u8(flags);
        msgs.zeros(3);
        msgs.add(body);
        msgs.zeros(n - body.size());
        ++count;
    }
    Bytes encode() const {
        Bytes o;
        o.u8(1);                                 /* version */
        o.u8(0);
        o.u16(count);
        o.u32(1);                                /* reference count */
        o.u32((uint32_t)msgs.size());
        o.zeros(4);                              /* messages start 8-byte aligned */
        o.add(msgs);
        return o;
    }
};

Bytes attribute(const std::string &name, double v) {
    const Bytes t = float_type(8), s = dataspace(0, nullptr);
    Bytes a;
    a.u8(1);
    a.u8(0);
    a.u16((unsigned)name.size() + 1);
    a.u16((unsigned)t.size());
    a.u16((unsigned)s.size());
    a.raw(name.c_str(), name.size() + 1);
    a.align8();
    a.add(t);
    a.align8();
    a.add(s);
    a.align8();
    uint64_t bits;
    std::memcpy(&bits, &v, 8);
    a.u64(bits);
    return a;
}

struct Geometry {
    int rank;
    uint64_t dims[3], chunk[3];
    uint64_t nchunk[3];     /* chunks per axis */
    uint64_t total;         /* chunks */
    size_t chunk_elems;
};

/* the dataset object header; btree = address of the chunk index root */
Bytes dataset_header(const Geometry &g, int level, uint64_t btree) {
    Header h;
    h.add(MSG_DATASPACE, 0, dataspace(g.rank, g.dims));
    h.add(MSG_DATATYPE, MSG_CONSTANT, float_type(4));
    Bytes fill;                                  /* version 2: incremental allocation, write if set, default */
    fill.u8(2); fill.u8(3); fill.u8(2); fill.u8(1); fill.u32(0);
    h.add(MSG_FILL, MSG_CONSTANT, fill);
    Bytes pl;                                    /* version 1: shuffle (element size), deflate (level) */
    pl.u8(1); pl.u8(2); pl.zeros(6);
    const struct { unsigned id; const char *name; uint32_t cd; } filters[2] = {
        {FILTER_SHUFFLE, "shuffle", 4}, {FILTER_DEFLATE, "deflate", (uint32_t)level}};
    for (const auto &f : filters) {
        const size_t nl = pad8(std::strlen(f.name) + 1);
        pl.u16(f.id);
        pl.u16((unsigned)nl);
        pl.u16(1);                               /* optional */
        pl.u16(1);                               /* one client value */
        pl.raw(f.name, std::strlen(f.name));
        pl.zeros(nl - std::strlen(f.name));
        pl.u32(f.cd);
        pl.u32(0);                               /* odd count of client values: pad */
    }
    h.add(MSG_PIPELINE, MSG_CONSTANT, pl);
    Bytes lay;                                   /* version 3, chunked */
    lay.u8(3); lay.u8(2); lay.u8(g.rank + 1);
    lay.u64(btree);
    for (int a = 0; a < g.rank; ++a) lay.u32((uint32_t)g.chunk[a]);
    lay.u32(4);                                  /* element size */
    h.add(MSG_LAYOUT, MSG_CONSTANT, lay);
    return h.encode();
}

/* a chunk as the B-tree keys it: stored size, filter mask, element offset */
struct ChunkKey {
    uint32_t size = 0, mask = 0;
    uint64_t off[3] = {0, 0, 0};
};

class File {
  public:
    explicit File(const char *path) : f_(std::fopen(path, "wb")) {}
    ~File() { if (f_) std::fclose(f_); }
    bool ok() const { return f_ && !bad_; }
    uint64_t pos() const { return pos_; }
    void write(const void *p, size_t n) {
        if (!f_ || bad_) return;
        if (n && std::fwrite(p, 1, n, f_) != n) bad_ = true;
        pos_ += n;
    }
    void write(const Bytes &b) { write(b.b.data(), b.size()); }
    void write_at(uint64_t at, const Bytes &b) {
        if (!f_ || bad_) return;
        if (fseeko(f_, (off_t)at, SEEK_SET) != 0) { bad_ = true; return; }
        if (b.size() && std::fwrite(b.b.data(), 1, b.size(), f_) != b.size()) bad_ = true;
        if (fseeko(f_, (off_t)pos_, SEEK_SET) != 0) bad_ = true;
    }
    bool close() {
        if (!f_) return false;
        const bool good = !bad_ && std::fclose(f_) == 0;
        f_ = nullptr;
        return good;
    }

  private:
    FILE *f_;
    bool bad_ = false;
    uint64_t pos_ = 0;
};

/* version-1 B-tree node of type 1 over `n` children with keys[0..n] */
Bytes chunk_node(const Geometry &g, int level, const uint64_t *child, const ChunkKey *keys, int n, uint64_t left,
                 uint64_t right) {
    Bytes b;
    b.raw("TREE", 4);
    b.u8(1);
    b.u8(level);
    b.u16(n);
    b.u64(left);
    b.u64(right);
    auto key = [&](const ChunkKey &k) {
        b.u32(k.size);
        b.u32(k.mask);
        for (int a = 0; a < g.rank; ++a) b.u64(k.off[a]);
        b.u64(0);                                /* the element-size dimension */
    };
    for (int i = 0; i < n; ++i) {
        key(keys[i]);
        b.u64(child[i]);
    }
    key(keys[n]);
    const size_t key_bytes = 8 + 8 * (size_t)(g.rank + 1);
    const size_t full = 24 + (2 * CHUNK_K + 1) * key_bytes + 2 * CHUNK_K * 8;
    b.zeros(full - b.size());                    /* readers load whole nodes */
    return b;
}

/* Writes the chunk index for `n` chunks (keys[0..n], addresses addr[0..n-1])
 * at the file's end; returns the root's address. */
uint64_t write_chunk_index(File &f, const Geometry &g, std::vector<ChunkKey> keys, std::vector<uint64_t> addr) {
    int level = 0;
    for (;;) {
        const size_t n = addr.size();
        const size_t nodes = (n + 2 * CHUNK_K - 1) / (2 * CHUNK_K);
        const size_t key_bytes = 8 + 8 * (size_t)(g.rank + 1);
        const size_t node_bytes = 24 + (2 * CHUNK_K + 1) * key_bytes + 2 * CHUNK_K * 8;
        const uint64_t first = f.pos();
        std::vector<ChunkKey> up_keys;
        std::vector<uint64_t> up_addr;
        for (size_t j = 0; j < nodes; ++j) {
            const size_t b = j * 2 * CHUNK_K, e = std::min(n, b + 2 * CHUNK_K);
            const uint64_t self = first + j * node_bytes;
            const uint64_t left = j ? self - node_bytes : UNDEF, right = j + 1 < nodes ? self + node_bytes : UNDEF;
            f.write(chunk_node(g, level, &addr[b], &keys[b], (int)(e - b), left, right));
            up_keys.push_back(keys[b]);
            up_addr.push_back(self);
        }
        up_keys.push_back(keys[n]);
        if (nodes == 1) return first;
        keys.swap(up_keys);
        addr.swap(up_addr);
        ++level;
    }
}

/* gathers chunk `c` of `data` (edge chunks padded with 0) and shuffles its bytes */
void gather_shuffled(const Geometry &g, const float *data, uint64_t c, std::vector<float> &tmp,
                     std::vector<uint8_t> &out, uint64_t origin[3]) {
    uint64_t q = c;
    for (int a = g.rank - 1; a >= 0; --a) {
        origin[a] = (q % g.nchunk[a]) * g.chunk[a];
        q /= g.nchunk[a];
    }
    uint64_t D[3] = {1, 1, 1}, C[3] = {1, 1, 1}, O[3] = {0, 0, 0};
    for (int a = 0; a < g.rank; ++a) {
        D[3 - g.rank + a] = g.dims[a];
        C[3 - g.rank + a] = g.chunk[a];
        O[3 - g.rank + a] = origin[a];
    }
    std::fill(tmp.begin(), tmp.end(), 0.0f);
    const uint64_t n2 = std::min(C[2], D[2] - O[2]);
    for (uint64_t i0 = 0; i0 < C[0] && O[0] + i0 < D[0]; ++i0)
        for (uint64_t i1 = 0; i1 < C[1] && O[1] + i1 < D[1]; ++i1)
            std::memcpy(&tmp[(i0 * C[1] + i1) * C[2]], &data[((O[0] + i0) * D[1] + O[1] + i1) * D[2] + O[2]],
                        n2 * sizeof(float));
    const size_t m = g.chunk_elems;
    const uint8_t *src = (const uint8_t *)tmp.data();
    for (size_t e = 0; e < m; ++e)
        for (int j = 0; j < 4; ++j) out[j * m + e] = src[4 * e + j];
}

int write_file(const char *path, const Geometry &g, int nsets, const char *const *names, const float *const *data,
               int nattrs, const char *const *attr_names, const double *attr_values, int level, int threads,
               std::string &why) {
    /* link names in strcmp order (symbol-table nodes are searched by name) */
    std::vector<int> order(nsets);
    for (int s = 0; s < nsets; ++s) order[s] = s;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return std::strcmp(names[a], names[b]) < 0; });
    for (int s = 1; s < nsets; ++s)
        if (!std::strcmp(names[order[s]], names[order[s - 1]])) {
            why = std::string("dataset name given twice: ") + names[order[s]];
            return CB_EINVAL;
        }
    Bytes heap_data;
    heap_data.zeros(8);                          /* offset 0: the empty name */
    std::vector<uint64_t> name_off(nsets);
    for (int s = 0; s < nsets; ++s) {
        name_off[order[s]] = heap_data.size();
        heap_data.raw(names[order[s]], std::strlen(names[order[s]]) + 1);
        heap_data.align8();
    }

    /* metadata block: superblock, root header, heap, group B-tree, symbol-table node, dataset headers */
    auto root_header = [&](uint64_t btree, uint64_t heap) {
        Header h;
        Bytes st;
        st.u64(btree);
        st.u64(heap);
        h.add(MSG_SYMBOL_TABLE, MSG_CONSTANT, st);
        for (int i = 0; i < nattrs; ++i) h.add(MSG_ATTRIBUTE, 0, attribute(attr_names[i], attr_values[i]));
        return h.encode();
    };
    const size_t root_bytes = root_header(0, 0).size();
    const size_t heap_hdr_bytes = 32;
    const size_t gtree_bytes = 24 + (2 * GROUP_INTERNAL_K + 1) * 8 + 2 * GROUP_INTERNAL_K * 8;
    const size_t snod_bytes = 8 + 2 * GROUP_LEAF_K * ENTRY_BYTES;
    const size_t ds_bytes = dataset_header(g, level, 0).size();
    const uint64_t a_root = SUPERBLOCK_BYTES;
    const uint64_t a_heap = a_root + root_bytes;
    const uint64_t a_heap_data = a_heap + heap_hdr_bytes;
    const uint64_t a_gtree = a_heap_data + heap_data.size();
    const uint64_t a_snod = a_gtree + gtree_bytes;
    const uint64_t a_ds0 = a_snod + snod_bytes;
    const uint64_t meta_bytes = a_ds0 + (uint64_t)nsets * ds_bytes;

    File f(path);
    if (!f.ok()) {
        why = std::string("cannot open ") + path + " for writing";
        return CB_EIO;
    }
    {
        Bytes z;
        z.zeros(meta_bytes);
        f.write(z);
    }

    /* chunks, dataset by dataset, then each dataset's chunk index */
    const size_t raw_bytes = g.chunk_elems * sizeof(float);
    const int T = threads > 0 ? threads : omp_get_max_threads();
    const uint64_t batch = (uint64_t)std::max(1, T) * 4;
    std::vector<uint64_t> btree(nsets);
    int zfail = 0;
    for (int s = 0; s < nsets && f.ok() && !zfail; ++s) {
        std::vector<ChunkKey> keys(g.total + 1);
        std::vector<uint64_t> addr(g.total);
        for (uint64_t b0 = 0; b0 < g.total && f.ok() && !zfail; b0 += batch) {
            const int64_t nb = (int64_t)std::min(batch, g.total - b0);
            std::vector<std::vector<uint8_t>> out(nb);
#pragma omp parallel num_threads(T)
            {
                std::vector<float> tmp(g.chunk_elems);
                std::vector<uint8_t> shuf(raw_bytes);
#pragma omp for schedule(dynamic, 1)
                for (int64_t i = 0; i < nb; ++i) {
                    ChunkKey &k = keys[b0 + i];
                    gather_shuffled(g, data[s], b0 + i, tmp, shuf, k.off);
                    uLongf len = compressBound((uLong)raw_bytes);
                    out[i].resize(len);
                    const int zs = compress2(out[i].data(), &len, shuf.data(), (uLong)raw_bytes, level);
                    if (zs != Z_OK) {
#pragma omp atomic write
                        zfail = 1;
                        continue;
                    }
                    if (len <= raw_bytes) {
                        out[i].resize(len);
                        k.mask = 0;
                    } else {
                        out[i].assign(shuf.begin(), shuf.end());
                        k.mask = 1u << 1;        /* deflate (second filter) not applied */
                    }
                    k.size = (uint32_t)out[i].size();
                }
            }
            for (int64_t i = 0; i < nb && !zfail; ++i) {
                addr[b0 + i] = f.pos();
                f.write(out[i].data(), out[i].size());
            }
        }
        if (zfail) break;
        ChunkKey &end = keys[g.total];           /* just past the last chunk */
        for (int a = 0; a < g.rank; ++a) end.off[a] = keys[g.total - 1].off[a] + g.chunk[a];
        btree[s] = write_chunk_index(f, g, keys, addr);
    }
    if (zfail) {
        why = "zlib compress2 failed";
        return CB_EIO;
    }
    const uint64_t eof = f.pos();

    Bytes meta;
    meta.raw("\x89HDF\r\n\x1a\n", 8);
    meta.u8(0); meta.u8(0); meta.u8(0); meta.u8(0);   /* superblock, free space, root entry, reserved */
    meta.u8(0); meta.u8(8); meta.u8(8); meta.u8(0);   /* shared headers, offset and length sizes */
    meta.u16(GROUP_LEAF_K);
    meta.u16(GROUP_INTERNAL_K);
    meta.u32(0);                                      /* consistency flags */
    meta.u64(0);                                      /* base address */
    meta.u64(UNDEF);                                  /* free-space info */
    meta.u64(eof);
    meta.u64(UNDEF);                                  /* driver info */
    meta.u64(0);                                      /* root entry: name offset, header, cache type 1 */
    meta.u64(a_root);
    meta.u32(1);
    meta.u32(0);
    meta.u64(a_gtree);
    meta.u64(a_heap);
    meta.add(root_header(a_gtree, a_heap));
    meta.raw("HEAP", 4);
    meta.u8(0);
    meta.zeros(3);
    meta.u64(heap_data.size());
    meta.u64(1);                                      /* no free block */
    meta.u64(a_heap_data);
    meta.add(heap_data);
    const size_t gtree_at = meta.size();
    meta.raw("TREE", 4);
    meta.u8(0);                                       /* group node */
    meta.u8(0);                                       /* leaf */
    meta.u16(1);
    meta.u64(UNDEF);
    meta.u64(UNDEF);
    meta.u64(0);                                      /* key 0: the empty name */
    meta.u64(a_snod);
    meta.u64(nsets ? name_off[order[nsets - 1]] : 0); /* key 1: the last name */
    meta.zeros(gtree_at + gtree_bytes - meta.size());
    const size_t snod_at = meta.size();
    meta.raw("SNOD", 4);
    meta.u8(1);
    meta.u8(0);
    meta.u16(nsets);
    for (int s = 0; s < nsets; ++s) {
        meta.u64(name_off[order[s]]);
        meta.u64(a_ds0 + (uint64_t)order[s] * ds_bytes);
        meta.u32(0);                                  /* no cached scratch data */
        meta.u32(0);
        meta.zeros(16);
    }
    meta.zeros(snod_at + snod_bytes - meta.size());
    for (int s = 0; s < nsets; ++s) meta.add(dataset_header(g, level, btree[s]));
    if (meta.size() != meta_bytes) {
        why = "internal error: metadata size";
        return CB_EIO;
    }
    f.write_at(0, meta);
    if (!f.close()) {
        why = std::string("writing ") + path + " failed";
        return CB_EIO;
    }
    return CB_OK;
}

/* OutField's datasets and attributes, on the host, ready to write */
int prepare_snapshot(cb_handle *h, const char *path, int threads, cb::Snapshot &snap) {
    const int D = h->p.d, n = h->p.n_grids;
    /* bubble.cpp:891-895: thinning of large lattices */
    int reduc = 1;
    if (D == 2 && n > 2048) reduc = n / 2048;
    if (D == 3 && n > 512) reduc = n / 512;
    const int m = (n + reduc - 1) / reduc;
    const bool local = h->p.memorysave != 1;
    auto &full = snap.fields;
    full.assign(local ? 5 : 2, std::vector<float>(h->N));
    int r = cb_get_fields_f32(h, full[0].data(), full[1].data(), local ? full[2].data() : nullptr,
                              local ? full[3].data() : nullptr, local ? full[4].data() : nullptr);
    if (r != CB_OK) return r;
    if (reduc > 1) {
        /* bubble.cpp:905-915: every reduc-th point per axis, in lattice order */
        const size_t n0 = D >= 3 ? (size_t)n : 1, n1 = D >= 2 ? (size_t)n : 1;
        const size_t s0 = D >= 3 ? reduc : 1, s1 = D >= 2 ? reduc : 1;
        for (auto &v : full) {
            size_t count = 0;
            for (size_t i0 = 0; i0 < n0; i0 += s0)
                for (size_t i1 = 0; i1 < n1; i1 += s1)
                    for (size_t i2 = 0; i2 < (size_t)n; i2 += reduc) v[count++] = v[(i0 * n1 + i1) * n + i2];
            v.resize(count);
            v.shrink_to_fit();
        }
    }
    /* bubble.cpp:934-940: shape (m,)*D; chunks of the whole field (1-D), rows (2-D), planes (3-D) */
    snap.D = D;
    for (int a = 0; a < 3; ++a) snap.dims[a] = snap.chunk[a] = m;
    if (D == 2) snap.chunk[0] = std::min<int64_t>(m, std::max<int64_t>(1, 65536 / m));
    if (D == 3) snap.chunk[0] = 1;
    cb_sums s;
    if ((r = cb_get_sums(h, &s)) != CB_OK) return r;
    /* bubble.cpp:945-951: D, L, nGrids, reduc, c, t, a */
    const double av[7] = {(double)D, h->p.L, (double)n, (double)reduc, h->p.c, s.t, s.a};
    std::copy(av, av + 7, snap.attrs);
    snap.path = path;
    snap.threads = threads;
    return CB_OK;
}

int write_snapshot(const cb::Snapshot &snap, std::string &err) {
    static const char *names[5] = {"phi", "pi", "Ekin", "gradphi", "potEnergy"};
    static const char *an[7] = {"D", "L", "nGrids", "reduc", "c", "t", "a"};
    const float *data[5];
    for (size_t f = 0; f < snap.fields.size(); ++f) data[f] = snap.fields[f].data();
    const int r = cb_h5_write_floats(snap.path.c_str(), snap.D, snap.dims, snap.chunk, (int)snap.fields.size(),
                                     names, data, 7, an, snap.attrs, 9, snap.threads);
    if (r != CB_OK) err = cb_last_error(nullptr);
    return r;
}

}  // namespace

namespace cb {
int finish_writer(cb_handle *h) {
    if (!h->writer) return CB_OK;
    if (h->writer->th.joinable()) h->writer->th.join();
    const int r = h->writer->status;
    const std::string e = h->writer->err;
    delete h->writer;
    h->writer = nullptr;
    return r == CB_OK ? CB_OK : fail(h, r, e);
}
}  // namespace cb

extern "C" {

int cb_h5_write_floats(const char *path, int rank, const int64_t *dims, const int64_t *chunk, int nsets,
                       const char *const *names, const float *const *data, int nattrs,
                       const char *const *attr_names, const double *attr_values, int deflate_level, int threads) {
    return cb::guard(nullptr, [&]() -> int {
        if (!path || !dims || !chunk) return fail(nullptr, CB_EINVAL, "path, dims and chunk must not be NULL");
        if (rank < 1 || rank > 3) return fail(nullptr, CB_EINVAL, "rank must be 1, 2 or 3");
        if (nsets < 0 || nsets > MAX_SETS) return fail(nullptr, CB_EINVAL, "between 0 and 8 datasets");
        if (nattrs < 0 || (nattrs && (!attr_names || !attr_values)))
            return fail(nullptr, CB_EINVAL, "attribute names and values must not be NULL");
        if (nsets && (!names || !data)) return fail(nullptr, CB_EINVAL, "dataset names and data must not be NULL");
        if (deflate_level < 0 || deflate_level > 9) return fail(nullptr, CB_EINVAL, "deflate level must be 0..9");
        Geometry g{};
        g.rank = rank;
        g.total = 1;
        g.chunk_elems = 1;
        for (int a = 0; a < rank; ++a) {
            if (dims[a] < 1 || chunk[a] < 1 || chunk[a] > dims[a])
                return fail(nullptr, CB_EINVAL, "dims must be >= 1 and 1 <= chunk <= dims");
            g.dims[a] = (uint64_t)dims[a];
            g.chunk[a] = (uint64_t)chunk[a];
            g.nchunk[a] = (g.dims[a] + g.chunk[a] - 1) / g.chunk[a];
            g.total *= g.nchunk[a];
            g.chunk_elems *= (size_t)g.chunk[a];
        }
        if (g.chunk_elems * sizeof(float) >= (size_t(1) << 32)) return fail(nullptr, CB_EINVAL, "chunk of 4 GiB or more");
        for (int s = 0; s < nsets; ++s)
            if (!names[s] || !names[s][0] || !data[s]) return fail(nullptr, CB_EINVAL, "empty dataset name or NULL data");
        for (int i = 0; i < nattrs; ++i)
            if (!attr_names[i] || !attr_names[i][0]) return fail(nullptr, CB_EINVAL, "empty attribute name");
        std::string why;
        const int r = write_file(path, g, nsets, names, data, nattrs, attr_names, attr_values, deflate_level, threads, why);
        if (r != CB_OK) return fail(nullptr, r, why);
        return CB_OK;
    });
}

int cb_out_field(cb_handle *h, const char *path, int threads) {
    return cb::guard(h, [&]() -> int {
        if (!h || !path) return fail(h, CB_EINVAL, "handle and path must not be NULL");
        if (h->writer) return fail(h, CB_EBUSY, "a snapshot write is in flight (cb_out_field_wait first)");
        cb::Snapshot snap;
        int r = prepare_snapshot(h, path, threads, snap);
        if (r != CB_OK) return r;
        std::string err;
        r = write_snapshot(snap, err);
        return r == CB_OK ? CB_OK : fail(h, r, err);
    });
}

int cb_out_field_async(cb_handle *h, const char *path, int threads) {
    return cb::guard(h, [&]() -> int {
        if (!h || !path) return fail(h, CB_EINVAL, "handle and path must not be NULL");
        if (h->writer) return fail(h, CB_EBUSY, "a snapshot write is in flight (cb_out_field_wait first)");
        auto snap = std::make_shared<cb::Snapshot>();
        /* leave one host thread to the caller, who keeps launching steps */
        if (threads <= 0) threads = std::max(1, omp_get_max_threads() - 1);
        int r = prepare_snapshot(h, path, threads, *snap);
        if (r != CB_OK) return r;
        auto *w = new cb::SnapshotWriter;
        try {
            w->th = std::thread([w, snap] { w->status = write_snapshot(*snap, w->err); });
        } catch (...) {
            delete w;
            return fail(h, CB_ENOMEM, "cannot start the snapshot writer thread");
        }
        h->writer = w;
        return CB_OK;
    });
}

int cb_out_field_wait(cb_handle *h) {
    if (!h) return fail(nullptr, CB_EINVAL, "handle is NULL");
    return cb::finish_writer(h);
}

}  // extern "C"
