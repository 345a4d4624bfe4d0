// ref_dump.cu -- golden-vector harness around the reference's OWN analysis.
//
// Built by oracle/Makefile against the reference sources where they lie
// (-I <reference>/recblock-sptrsv, csrsv2_shim.h force-included); the binary
// goes to oracle/_ref/.  It runs get_recblock_size + L_/U_preprocessing
// (recblocking_preprocess.h:298-385, 387-967, 969-1474) exactly as
// recblocking_solver (recblocking_solver.h:69-103) calls them, on a CSC read
// from a file, and writes every integer output plus the packed values.
// Device calls inside the reference's analysis fail harmlessly on a host
// without a GPU; the integer analysis is computed on the host either way.
//
// Input : int32 m, nnz, substitution, lv; int32 colptr[m+1]; int32 rowidx[nnz]; f64 val[nnz]
// Output: records {char name[32]; int32 kind (0=int32,1=f64); int64 count; data}
#include "recblocking_preprocess.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

static FILE *g_out;

static void put_i(const char *name, const int *p, long long n) {
    char nm[32] = {0};
    strncpy(nm, name, 31);
    int32_t kind = 0;
    int64_t cnt = n;
    fwrite(nm, 1, 32, g_out);
    fwrite(&kind, 4, 1, g_out);
    fwrite(&cnt, 8, 1, g_out);
    if (n) fwrite(p, 4, (size_t)n, g_out);
}
static void put_d(const char *name, const double *p, long long n) {
    char nm[32] = {0};
    strncpy(nm, name, 31);
    int32_t kind = 1;
    int64_t cnt = n;
    fwrite(nm, 1, 32, g_out);
    fwrite(&kind, 4, 1, g_out);
    fwrite(&cnt, 8, 1, g_out);
    if (n) fwrite(p, 8, (size_t)n, g_out);
}

int main(int argc, char **argv) {
    if (argc != 3) {
        fprintf(stderr, "usage: ref_dump <in.bin> <out.bin>\n");
        return 2;
    }
    FILE *f = fopen(argv[1], "rb");
    if (!f) return 3;
    int32_t hdr[4];
    if (fread(hdr, 4, 4, f) != 4) return 4;
    int m = hdr[0], nnz = hdr[1], substitution = hdr[2], lv = hdr[3];
    int n = m;
    std::vector<int> colptr(m + 1), rowidx(nnz);
    std::vector<double> val(nnz);
    if (fread(colptr.data(), 4, m + 1, f) != (size_t)(m + 1)) return 4;
    if (fread(rowidx.data(), 4, nnz, f) != (size_t)nnz) return 4;
    if (fread(val.data(), 8, nnz, f) != (size_t)nnz) return 4;
    fclose(f);

    // recblocking_solver.h:30-67 set-up
    int tri_block = 1 << lv, squ_block = tri_block - 1, sum_block = tri_block + squ_block;
    std::vector<SpTRSV_block> trsv(tri_block);
    std::vector<SpMV_block> mv(squ_block > 0 ? squ_block : 1);
    memset(trsv.data(), 0, sizeof(SpTRSV_block) * trsv.size());
    memset(mv.data(), 0, sizeof(SpMV_block) * mv.size());
    for (int i = 0; i < squ_block; i++) mv[i].method = -1;
    std::vector<int> blk_m(sum_block), blk_n(sum_block), blk_nnz(sum_block);
    std::vector<int> loc_off(sum_block, 0), tmp_off(sum_block, 0), levelItem(m);
    std::vector<int> stu(sum_block, -1), std_(sum_block, -1), sru(sum_block, -1), srd(sum_block, -1),
        srr(sum_block, -1), srl(sum_block, -1);
    int ptr_size = 1, idx_size = 0, dcsr_size = 0;
    std::vector<int> cp_new(n + 1), ri_new(nnz);
    std::vector<double> va_new(nnz);

    get_recblock_size(rowidx.data(), colptr.data(), val.data(), ri_new.data(), cp_new.data(), va_new.data(),
                      nnz, m, n, levelItem.data(), substitution, lv, loc_off.data(), tmp_off.data(),
                      blk_m.data(), blk_n.data(), blk_nnz.data(), stu.data(), std_.data(), sru.data(),
                      srd.data(), srr.data(), srl.data(), &ptr_size, &idx_size, &dcsr_size);

    std::vector<int> Ptr(ptr_size, 0), Index(idx_size > 0 ? idx_size : 1, 0), dcsr(dcsr_size > 0 ? dcsr_size : 1, 0);
    std::vector<double> Val(idx_size > 0 ? idx_size : 1, 0.0);
    std::vector<int> ptr_offset(sum_block + 1), index_offset(sum_block + 1), dcsr_offset(sum_block + 1);
    Ptr[0] = 0;
    ptr_offset[0] = 1;
    index_offset[0] = 0;
    dcsr_offset[0] = 0;
    if (substitution == SUBSTITUTION_FORWARD)
        L_preprocessing(ri_new.data(), cp_new.data(), va_new.data(), nnz, m, n, substitution, lv, blk_m.data(),
                        blk_n.data(), blk_nnz.data(), stu.data(), std_.data(), sru.data(), srd.data(), srr.data(),
                        srl.data(), mv.data(), trsv.data(), Ptr.data(), Index.data(), dcsr.data(), Val.data(),
                        ptr_offset.data(), index_offset.data(), dcsr_offset.data(), ptr_size, idx_size, dcsr_size);
    else
        U_preprocessing(ri_new.data(), cp_new.data(), va_new.data(), nnz, m, n, substitution, lv, blk_m.data(),
                        blk_n.data(), blk_nnz.data(), stu.data(), std_.data(), sru.data(), srd.data(), srr.data(),
                        srl.data(), mv.data(), trsv.data(), Ptr.data(), Index.data(), dcsr.data(), Val.data(),
                        ptr_offset.data(), index_offset.data(), dcsr_offset.data(), ptr_size, idx_size, dcsr_size);

    // Per-block method codes and level statistics.  Tri-block local level sets
    // come from the reference's findlevel (findlevel.h:7) on the block's CSC,
    // extracted with the bounds filter of recblocking_preprocess.h:439-451.
    std::vector<int> method(sum_block, -1), nlv(sum_block, 0), longrow(sum_block, 0), m_new(sum_block, -1);
    std::vector<int> lvl_ptr, lvl_item, m_lv, off_lv, nnz_lv;
    int ti = 0, si = 0;
    for (int b = 0; b < sum_block; ++b) {
        if ((b & 1) == 0) {
            SpTRSV_block &t = trsv[ti++];
            method[b] = t.method;
            int up = stu[b], down = std_[b], bm = blk_m[b];
            std::vector<int> scp(bm + 1, 0), sri;
            for (int c = up; c < down; ++c) {
                for (int k = cp_new[c]; k < cp_new[c + 1]; ++k) {
                    int r = ri_new[k];
                    bool keep = substitution == SUBSTITUTION_FORWARD ? r < down : r >= up;
                    if (keep) sri.push_back(r - up);
                }
                scp[c - up + 1] = (int)sri.size();
            }
            std::vector<int> rrp(bm + 1);
            matrix_transposition_litelite(bm, bm, (int)sri.size(), scp.data(), sri.data(), rrp.data());
            std::vector<int> lp(bm + 1), li(bm);
            int nl = 1;
            if (bm == (int)sri.size()) {
                lp[0] = 0;
                lp[1] = bm;
                for (int i = 0; i < bm; ++i) li[i] = i;
            } else {
                findlevel(scp.data(), sri.data(), rrp.data(), bm, &nl, lp.data(), li.data());
            }
            nlv[b] = nl;
            lvl_ptr.insert(lvl_ptr.end(), lp.begin(), lp.begin() + nl + 1);
            lvl_item.insert(lvl_item.end(), li.begin(), li.end());
            if (t.method == 2) {
                for (int l = 0; l < t.nlv; ++l) {
                    m_lv.push_back(t.m_lv_array[l]);
                    off_lv.push_back(t.offset_array[l]);
                    nnz_lv.push_back(t.nnz_lv_array[l]);
                }
            }
        } else {
            SpMV_block &s = mv[si++];
            method[b] = s.method;
            longrow[b] = s.method >= 0 ? s.longrow : 0;
            m_new[b] = (s.method == 1 || s.method == 3) ? s.m_new : -1;
        }
    }

    g_out = fopen(argv[2], "wb");
    if (!g_out) return 5;
    put_i("levelItem", levelItem.data(), m);
    put_i("loc_off", loc_off.data(), sum_block);
    put_i("tmp_off", tmp_off.data(), sum_block);
    put_i("blk_m", blk_m.data(), sum_block);
    put_i("blk_n", blk_n.data(), sum_block);
    put_i("blk_nnz", blk_nnz.data(), sum_block);
    put_i("subtri_up", stu.data(), sum_block);
    put_i("subtri_down", std_.data(), sum_block);
    put_i("subrec_up", sru.data(), sum_block);
    put_i("subrec_down", srd.data(), sum_block);
    put_i("subrec_right", srr.data(), sum_block);
    put_i("subrec_left", srl.data(), sum_block);
    int sizes[3] = {ptr_size, idx_size, dcsr_size};
    put_i("sizes", sizes, 3);
    put_i("ptr_offset", ptr_offset.data(), sum_block + 1);
    put_i("index_offset", index_offset.data(), sum_block + 1);
    put_i("dcsrindex_offset", dcsr_offset.data(), sum_block + 1);
    put_i("recblock_Ptr", Ptr.data(), ptr_offset[sum_block]);
    put_i("recblock_Index", Index.data(), index_offset[sum_block]);
    put_d("recblock_Val", Val.data(), index_offset[sum_block]);
    put_i("recblock_dcsr_rowidx", dcsr.data(), dcsr_offset[sum_block]);
    put_i("method", method.data(), sum_block);
    put_i("nlv", nlv.data(), sum_block);
    put_i("longrow", longrow.data(), sum_block);
    put_i("m_new_dcsr", m_new.data(), sum_block);
    put_i("lvl_ptr", lvl_ptr.data(), (long long)lvl_ptr.size());
    put_i("lvl_item", lvl_item.data(), (long long)lvl_item.size());
    put_i("m_lv", m_lv.data(), (long long)m_lv.size());
    put_i("offset_lv", off_lv.data(), (long long)off_lv.size());
    put_i("nnz_lv", nnz_lv.data(), (long long)nnz_lv.size());
    fclose(g_out);
    return 0;
}
