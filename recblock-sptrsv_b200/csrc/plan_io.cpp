// plan_io.cpp -- saving and loading an analysed plan (rbs_plan_save /
// rbs_plan_load): a warm start for resident factors, e.g. a serving process
// that restarts.  The file holds the plan's host side (scalars, options,
// the reference-format inputs kept for export, level order, labels, the
// execution blocks and every pool) in a versioned binary layout of this
// build, followed by a 64-bit digest of everything before it; the device
// state is rebuilt from it on load.  A file whose digest does not match is
// rejected, so a damaged plan never reaches the kernels (plan files are this
// library's own output: the digest guards against damage, not forgery).
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "rbs.h"
#include "lc_layout.h"
#include "rbs_internal.h"

namespace rbs {

namespace {

constexpr char kMagic[8] = {'R', 'B', 'S', 'P', 'L', 'A', 'N', '2'};

// The SplitMix64 output function (Steele, Lea and Flood, "Fast splittable
// pseudorandom number generators", OOPSLA 2014): a 64-bit mixing step.
inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// Digest of n bytes: 8-byte words folded through mix64 in 1 MB chunks (on
// host threads for large ranges), the chunk digests then folded in order.
uint64_t digest(const void *p, size_t n) {
    const unsigned char *b = static_cast<const unsigned char *>(p);
    constexpr size_t kChunk = size_t(1) << 20;
    const size_t nch = (n + kChunk - 1) / kChunk;
    std::vector<uint64_t> part(nch);
    auto one = [&](size_t c) {
        const size_t s = c * kChunk, e = std::min(n, s + kChunk);
        uint64_t h = mix64(0x9e3779b97f4a7c15ULL + c);
        size_t i = s;
        for (; i + 8 <= e; i += 8) {
            uint64_t w;
            std::memcpy(&w, b + i, 8);
            h = mix64(h ^ w);
        }
        if (i < e) {
            uint64_t w = 0;
            std::memcpy(&w, b + i, e - i);
            h = mix64(h ^ w ^ ((uint64_t)(e - i) << 56));
        }
        part[c] = h;
    };
    if (nch > 4)
        parallel_for(nch, one);
    else
        for (size_t c = 0; c < nch; ++c) one(c);
    uint64_t h = mix64(n);
    for (uint64_t x : part) h = mix64(h ^ x);
    return h;
}

struct Writer {
    FILE *f;
    bool ok = true;
    uint64_t sum = 0;  // digest of every byte written through pod/vec
    void fold(const void *p, size_t n) { sum = mix64(sum ^ digest(p, n)); }
    template <typename T>
    void pod(const T &v) {
        fold(&v, sizeof(T));
        ok = ok && std::fwrite(&v, sizeof(T), 1, f) == 1;
    }
    template <typename T, typename A>
    void vec(const std::vector<T, A> &v) {
        const uint64_t n = v.size();
        pod(n);
        if (n) {
            fold(v.data(), sizeof(T) * (size_t)n);
            ok = ok && std::fwrite(v.data(), sizeof(T), n, f) == n;
        }
    }
};

struct Reader {
    FILE *f;
    bool ok = true;
    uint64_t sum = 0;  // digest of every byte read through pod/vec
    void fold(const void *p, size_t n) { sum = mix64(sum ^ digest(p, n)); }
    template <typename T>
    void pod(T &v) {
        ok = ok && std::fread(&v, sizeof(T), 1, f) == 1;
        if (ok) fold(&v, sizeof(T));
    }
    template <typename T, typename A>
    void vec(std::vector<T, A> &v) {
        uint64_t n = 0;
        pod(n);
        if (!ok || n > (1ull << 40) / sizeof(T)) {
            ok = false;
            return;
        }
        v.resize((size_t)n);
        if (n) {
            ok = ok && std::fread(v.data(), sizeof(T), n, f) == n;
            if (ok) fold(v.data(), sizeof(T) * (size_t)n);
        }
    }
};

// One list of every plan field, used in both directions.
template <typename IO>
void fields(IO &io, Plan &P) {
    io.pod(P.n);
    io.pod(P.nnz);
    io.pod(P.lv);
    io.pod(P.sub);
    io.pod(P.nlevel);
    io.pod(P.sum_block);
    io.pod(P.step);
    io.pod(P.opt);
    io.pod(P.analyse_ms);
    io.pod(P.device_analyse_ms);
    io.pod(P.device_bfs);
    io.vec(P.in_cp);
    io.vec(P.in_ri);
    io.vec(P.in_va);
    io.vec(P.bfs_item);
    io.vec(P.bfs_ptr);
    io.vec(P.label);
    io.vec(P.perm);
    io.vec(P.blocks);
    io.vec(P.rp_pool);
    io.vec(P.col_pool);
    io.vec(P.lvl_pool);
    io.vec(P.map_pool);
    io.vec(P.rows_pool);
    io.vec(P.val_pool);
    io.vec(P.inv_diag);
    io.vec(P.band_coef);
    io.vec(P.band_inv);
    io.vec(P.ell_col);
    io.vec(P.ell_val);
    io.vec(P.ell_chunks);
    io.vec(P.ca_tab);
    io.vec(P.ca_col);
    io.vec(P.ca_val);
    io.vec(P.lc_rec64);
    io.vec(P.lc_rec32);
    io.vec(P.lc_tab);
    io.vec(P.lc_segs);
    io.vec(P.seg_rows);
    io.vec(P.dev_reorder_cp);
    io.vec(P.dev_reorder_ri);
    io.vec(P.full_rp);
    io.vec(P.full_col);
    io.vec(P.full_val);
}

// layout signature: a file is read only by a build with the same record
// sizes and the same constants that give the plan's arrays their meaning
// (the squares' row-length classes, the staged-level window, the level-chunk
// layout and its copy distance): a plan whose lists were cut at other
// thresholds would solve wrongly, not fail
uint64_t layout_signature() {
    const uint64_t c[] = {sizeof(ExecBlock), sizeof(rbs_options), sizeof(Plan), (uint64_t)SQ_MEDROW,
                          (uint64_t)SQ_LONGROW, (uint64_t)CA_WINDOW_ROWS, (uint64_t)LC_XW, (uint64_t)LC_NB,
                          (uint64_t)LC_D, (uint64_t)LC_RMAX, (uint64_t)LC_T, (uint64_t)LC_RING, (uint64_t)LC_FMAX,
                          (uint64_t)LC_HDR_INTS};
    uint64_t h = 0;
    for (uint64_t v : c) h = mix64(h ^ v);
    return h;
}

}  // namespace

int plan_save(const Plan &P, const char *path, std::string &err) {
    FILE *f = std::fopen(path, "wb");
    if (!f) {
        err = std::string("rbs_plan_save: cannot open ") + path;
        return RBS_ERR_ARG;
    }
    Writer w{f};
    w.ok = std::fwrite(kMagic, 1, sizeof(kMagic), f) == sizeof(kMagic);
    w.pod(layout_signature());
    fields(w, const_cast<Plan &>(P));
    const uint64_t sum = w.sum;
    w.ok = w.ok && std::fwrite(&sum, sizeof(sum), 1, f) == 1;
    const bool ok = w.ok && std::fclose(f) == 0;
    if (!ok) {
        err = std::string("rbs_plan_save: write failed: ") + path;
        return RBS_ERR_ARG;
    }
    return RBS_OK;
}

int plan_load(Plan &P, const char *path, std::string &err) {
    FILE *f = std::fopen(path, "rb");
    if (!f) {
        err = std::string("rbs_plan_load: cannot open ") + path;
        return RBS_ERR_ARG;
    }
    char magic[8] = {0};
    Reader r{f};
    r.ok = std::fread(magic, 1, sizeof(magic), f) == sizeof(magic) && std::memcmp(magic, kMagic, sizeof(kMagic)) == 0;
    uint64_t sig = 0;
    r.pod(sig);
    if (!r.ok || sig != layout_signature()) {
        std::fclose(f);
        err = std::string("rbs_plan_load: not a plan file of this build: ") + path;
        return RBS_ERR_ARG;
    }
    fields(r, P);
    uint64_t stored = 0;
    const bool have_sum = r.ok && std::fread(&stored, sizeof(stored), 1, f) == 1;
    const bool at_end = have_sum && std::fgetc(f) == EOF;
    std::fclose(f);
    if (!r.ok || !have_sum) {
        err = std::string("rbs_plan_load: truncated or corrupt plan file: ") + path;
        return RBS_ERR_ARG;
    }
    if (stored != r.sum || !at_end) {
        err = std::string("rbs_plan_load: plan file damaged (digest mismatch): ") + path;
        return RBS_ERR_ARG;
    }
    // consistency of the sizes the executor relies on
    const bool sane = P.n > 0 && P.nnz >= P.n && P.sum_block == (int)P.blocks.size() && P.sum_block == 2 * (1 << P.lv) - 1 &&
                      P.perm.size() == (size_t)P.n && P.full_rp.size() == (size_t)P.n + 1 &&
                      P.full_col.size() == (size_t)P.nnz && P.inv_diag.size() == (size_t)P.n;
    if (!sane) {
        err = std::string("rbs_plan_load: inconsistent plan file: ") + path;
        return RBS_ERR_ARG;
    }
    P.dev = nullptr;
    return RBS_OK;
}

}  // namespace rbs
