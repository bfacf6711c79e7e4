// .cbplan files: "CBPLAN\0\0", format version, a byte-order probe, the plan's
// options, then every field of the host CB structure(s) and device layout(s)
// in the fixed order of visit() below (scalars raw, arrays as a 64-bit count
// and raw elements), and a 64-bit checksum of everything after the header.
// The same visit() drives writing and reading, so the two cannot drift apart;
// adding a field means bumping kPlanFileVersion.
#include "cb_planfile.hpp"

#include <cstdio>
#include <cstring>
#include <type_traits>
#include <vector>

namespace cb {
namespace {

constexpr char kMagic[8] = {'C', 'B', 'P', 'L', 'A', 'N', 0, 0};
constexpr uint32_t kOrderProbe = 0x01020304u;

// 64-bit multiplicative hash over 8-byte words (tail bytes zero-padded)
struct Checksum {
    uint64_t h = 0x9e3779b97f4a7c15ull;
    uint8_t tail[8] = {};
    int ntail = 0;
    void word(uint64_t w) {
        h ^= w;
        h *= 0x100000001b3ull;
        h ^= h >> 29;
    }
    void add(const void *p, size_t n) {
        const uint8_t *b = static_cast<const uint8_t *>(p);
        while (n && ntail) {
            tail[ntail++] = *b++;
            --n;
            if (ntail == 8) {
                uint64_t w;
                std::memcpy(&w, tail, 8);
                word(w);
                ntail = 0;
            }
        }
        for (; n >= 8; n -= 8, b += 8) {
            uint64_t w;
            std::memcpy(&w, b, 8);
            word(w);
        }
        while (n--) tail[ntail++] = *b++;
    }
    uint64_t done() {
        if (ntail) {
            std::memset(tail + ntail, 0, 8 - ntail);
            uint64_t w;
            std::memcpy(&w, tail, 8);
            word(w);
            ntail = 0;
        }
        return h;
    }
};

struct Writer {
    std::FILE *f = nullptr;
    Checksum ck;
    bool ok = true;
    void raw(const void *p, size_t n) {
        if (ok && n && std::fwrite(p, 1, n, f) != n) ok = false;
        ck.add(p, n);
    }
    template <class T>
    void operator()(T &v) {
        static_assert(std::is_trivially_copyable<T>::value, "scalar field");
        raw(&v, sizeof(T));
    }
    template <class T>
    void operator()(std::vector<T> &v) {
        uint64_t n = v.size();
        raw(&n, sizeof n);
        raw(v.data(), n * sizeof(T));
    }
};

struct Reader {
    std::FILE *f = nullptr;
    uint64_t left = 0;  // bytes of the file not yet read
    Checksum ck;
    bool ok = true;
    void raw(void *p, size_t n) {
        if (!ok) return;
        if (n > left || (n && std::fread(p, 1, n, f) != n)) {
            ok = false;
            return;
        }
        left -= n;
        ck.add(p, n);
    }
    template <class T>
    void operator()(T &v) {
        raw(&v, sizeof(T));
    }
    template <class T>
    void operator()(std::vector<T> &v) {
        uint64_t n = 0;
        raw(&n, sizeof n);
        if (!ok || n > left / sizeof(T)) {  // a count the file cannot hold
            ok = false;
            return;
        }
        v.resize(n);
        raw(v.data(), n * sizeof(T));
    }
};

// lean: scalars only (an SpMV-only file)
template <class Ar>
void visit(Ar &ar, HostCB &g, bool lean) {
    ar(g.o.bs), ar(g.o.row_owned), ar(g.o.waves), ar(g.o.dense_sixteenths), ar(g.o.force_coo64);
    ar(g.m), ar(g.n), ar(g.nnz), ar(g.gb_m), ar(g.gb_n), ar(g.nnzb);
    ar(g.gather_flag), ar(g.direct), ar(g.compact), ar(g.balanced);
    ar(g.super_sparse), ar(g.analyzed), ar(g.ratio), ar(g.sd_before), ar(g.sd_after);
    ar(g.unit_values);
    if (lean) return;
    ar(g.gb_row), ar(g.gb_col), ar(g.nnz_blk), ar(g.type_blk), ar(g.gb_row_ptr);
    ar(g.seg_rows), ar(g.seg_begin), ar(g.seg_end), ar(g.seg_direct), ar(g.seg_uniform);
    ar(g.row_uniform), ar(g.flat_row_ptr), ar(g.flat_col), ar(g.pat_row_ptr), ar(g.pat_col);
    ar(g.pat_out_ptr), ar(g.pat_out_rows), ar(g.block_cols_offset), ar(g.block_cols);
    ar(g.bidx_origin), ar(g.bidx_end), ar(g.bidx_nnz), ar(g.nnzb_orig);
    ar(g.u32_off), ar(g.f64_off), ar(g.pay_u32), ar(g.pay_f64), ar(g.src_ptr), ar(g.src);
}

// lean: no per-value arrays (value offsets, coordinates, sources, slots)
template <class Ar>
void visit(Ar &ar, DeviceLayout &L, bool lean) {
    ar(L.bs), ar(L.f32), ar(L.unit), ar(L.gather), ar(L.m), ar(L.n), ar(L.gb_m);
    ar(L.tiles), ar(L.blocks), ar(L.payload), ar(L.block_cols);
    ar(L.slots), ar(L.split_rows), ar(L.max_row_tiles), ar(L.max_entries);
    ar(L.max_tile_bytes), ar(L.coo_share), ar(L.nvals), ar(L.alg_bytes);
    if (lean) return;
    ar(L.val_off), ar(L.val_row), ar(L.val_col), ar(L.vsrc_ptr), ar(L.vsrc);
    ar(L.input_slot);
}

template <class Ar>
void visit_body(Ar &ar, PlanImage &img) {
    ar(img.flags);
    const bool lean = (img.flags & kPlanSpmvOnly) != 0;
    for (int32_t &v : img.opts) ar(v);
    ar(img.has_t);
    for (int64_t &c : img.counts) ar(c);
    visit(ar, *img.host, lean);
    visit(ar, *img.A, lean);
    if (img.has_t) {
        visit(ar, *img.host_t, lean);
        visit(ar, *img.AT, lean);
    }
}

}  // namespace

std::string save_plan(const PlanImage &img_in, const std::string &path) {
    std::FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return "cannot open " + path + " for writing";
    PlanImage img = img_in;
    Writer w;
    w.f = f;
    const uint32_t head[2] = {kPlanFileVersion, kOrderProbe};
    bool ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(head, 4, 2, f) == 2;
    visit_body(w, img);
    const uint64_t sum = w.ck.done();
    ok = ok && w.ok && std::fwrite(&sum, 8, 1, f) == 1;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? "" : "write error on " + path;
}

std::string load_plan(const std::string &path, PlanImage &img) {
    std::FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return "cannot open " + path;
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    char magic[8];
    uint32_t head[2] = {0, 0};
    if (size < 24 || std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, kMagic, 8) != 0 ||
        std::fread(head, 4, 2, f) != 2) {
        std::fclose(f);
        return path + " is not a plan file";
    }
    if (head[1] != kOrderProbe) {
        std::fclose(f);
        return path + " was written on a machine of the other byte order";
    }
    if (head[0] != kPlanFileVersion) {
        std::fclose(f);
        return path + ": plan file version " + std::to_string(head[0]) + ", this library reads " +
               std::to_string(kPlanFileVersion);
    }
    Reader r;
    r.f = f;
    r.left = (uint64_t)size - 16 - 8;
    visit_body(r, img);
    uint64_t sum = 0;
    const bool tail_ok = std::fread(&sum, 8, 1, f) == 1;
    std::fclose(f);
    if (!r.ok || !tail_ok || r.left != 0) return path + " is truncated or corrupt";
    if (sum != r.ck.done()) return path + " fails its checksum (corrupt)";
    return "";
}

}  // namespace cb
