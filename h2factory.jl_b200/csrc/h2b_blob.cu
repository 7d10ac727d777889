// Map blob: a self-contained binary image of an h2b_map_desc, so that a core built once (by the
// Julia glue from an H2Factory core, or by any host) can be stored on disk and loaded by any
// process without rebuilding trees, plans, collections, transfers, couplings and near blocks.
//
// The reference has no on-disk format (an AbstractH2Core lives in a Julia session,
// src/maps/core.jl:1-60); the blob carries exactly the fields of the descriptor, which are the
// core's read-only data (core.jl) plus the four plans a workspace is built from
// (src/maps/workspace.jl:81-100).
//
// Layout (little endian, every record 8-byte aligned):
//   "H2BMAP01"                       8 bytes
//   uint64 nrecords
//   nrecords x { uint32 tag; uint32 elem_bytes; int64 count; payload; zero padding to 8 bytes }
// Record 0 holds the scalars (BlobScalars); the others the arrays in a fixed order, each tagged
// by its field. Every array length follows from the scalars or from a CSR array stored before
// it, and is checked on load; the loaded descriptor points into the caller's buffer (no copies)
// and then goes through the same validation as any other descriptor.

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "h2b_internal.cuh"

namespace {

constexpr char kMagic[8] = {'H', '2', 'B', 'M', 'A', 'P', '0', '1'};

struct BlobSide {
    int32_t nnodes, nlevels, root, ndofs, agg_nstages, dis_nstages;
    int64_t coll_len, transfer_len;
};

struct BlobScalars {
    int32_t field, precision, ncomp, dim, nsectors, transfer_kind, coupling_kind, conj_leaf_adjoint;
    double alpha[3][2];
    int64_t ncouplings, coupling_len;
    int32_t near_nrows, near_kind;
    int64_t near_len;
    double near_wavenumber;
    int64_t coupling_perm_len;
    int32_t has_perm, pad;
    BlobSide side[2];
};

h2b_status err(h2b_status st, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return h2b::set_error_text(st, buf);
}

// One array of the descriptor: its tag, element size, pointer member, and length -- fixed, or
// the end of a CSR array (csr[ncsr]) that precedes it in the list.
struct Field {
    uint32_t tag, elem;
    const void **ptr;
    int64_t fixed;              // >= 0: required length
    const int32_t *const *csr;  // else: length = (*csr)[ncsr]
    int64_t ncsr;
};

std::vector<Field> fields(h2b_map_desc &d, bool has_perm) {
    std::vector<Field> f;
    const int fw = d.field == H2B_COMPLEX ? 2 : 1;
    auto fix = [&](uint32_t tag, uint32_t elem, const void *p, int64_t n) {
        f.push_back({tag, elem, (const void **)p, n > 0 ? n : 0, nullptr, 0});
    };
    auto dep = [&](uint32_t tag, uint32_t elem, const void *p, const int32_t *const *csr, int64_t n) {
        f.push_back({tag, elem, (const void **)p, -1, csr, n});
    };
    for (int si = 0; si < 2; ++si) {
        h2b_side_desc &s = si == 0 ? d.test : d.trial;
        const uint32_t b = 100 + 40 * si;
        const int64_t nn = s.nnodes;
        fix(b + 0, 4, &s.level, nn);
        fix(b + 1, 4, &s.parent, nn);
        fix(b + 2, 4, &s.sector, nn);
        fix(b + 3, 4, &s.child_ptr, nn + 1);
        dep(b + 4, 4, &s.child, &s.child_ptr, nn);
        fix(b + 5, 4, &s.value_ptr, nn + 1);
        dep(b + 6, 4, &s.value, &s.value_ptr, nn);
        fix(b + 7, 4, &s.shape, (int64_t)(s.nlevels + 1) * 3);
        fix(b + 8, 4, &s.agg_level, s.agg_nstages);
        fix(b + 9, 4, &s.agg_ptr, s.agg_nstages + 1);
        dep(b + 10, 4, &s.agg_node, &s.agg_ptr, s.agg_nstages);
        fix(b + 11, 1, &s.agg_store, nn);
        fix(b + 12, 4, &s.dis_level, s.dis_nstages);
        fix(b + 13, 4, &s.dis_ptr, s.dis_nstages + 1);
        dep(b + 14, 4, &s.dis_node, &s.dis_ptr, s.dis_nstages);
        fix(b + 15, 1, &s.dis_isnode, nn);
        fix(b + 16, 4, &s.i2o_ptr, nn + 1);
        dep(b + 17, 4, &s.i2o_src, &s.i2o_ptr, nn);
        dep(b + 18, 8, &s.i2o_coupling, &s.i2o_ptr, nn);
        fix(b + 19, 8, &s.coll_offset, nn);
        fix(b + 20, 8, &s.coll, s.coll_len * fw);  // lengths in field scalars
        fix(b + 21, 8, &s.transfer_offset, (int64_t)(s.nlevels + 1) * d.nsectors);
        fix(b + 22, 8, &s.transfer, s.transfer_len * fw);
    }
    fix(10, 8, &d.coupling_offset, d.ncouplings);
    fix(11, 8, &d.coupling, d.coupling_len);
    fix(12, 4, &d.near_row, d.near_nrows);
    fix(13, 4, &d.near_ptr, d.near_nrows + 1);
    dep(14, 4, &d.near_col, &d.near_ptr, d.near_nrows);
    if (d.near_kind == H2B_NEAR_STORED) {
        dep(15, 8, &d.near_offset, &d.near_ptr, d.near_nrows);
        fix(16, 8, &d.near, d.near_len * fw);
    } else {
        fix(17, 8, &d.test_points, (int64_t)d.test.ndofs * 3);
        fix(18, 8, &d.trial_points, (int64_t)d.trial.ndofs * 3);
    }
    if (has_perm) {
        fix(19, 8, &d.coupling_rowperm, d.ncouplings);
        fix(20, 8, &d.coupling_colperm, d.ncouplings);
        fix(21, 4, &d.coupling_perm, d.coupling_perm_len);
    }
    return f;
}

// required length of `f` under the pointers set so far; -1 if its CSR array is missing or bad
int64_t length_of(const Field &f) {
    if (f.fixed >= 0) return f.fixed;
    const int32_t *csr = *f.csr;
    if (!csr || f.ncsr < 0) return -1;
    return csr[f.ncsr] >= 0 ? csr[f.ncsr] : -1;
}

size_t pad8(size_t n) { return (n + 7) & ~size_t(7); }

}  // namespace

extern "C" {

h2b_status h2b_map_blob_write(const h2b_map_desc *desc, void *buf, size_t cap, size_t *size) {
    if (!desc || !size) return err(H2B_ERR_INVALID, "h2b_map_blob_write: NULL argument");
    if (desc->near_kind == H2B_NEAR_STORED && desc->near_on_device)
        return err(H2B_ERR_INVALID, "h2b_map_blob_write: near blocks must be in host memory");
    h2b_map_desc d = *desc;
    const bool has_perm = d.coupling_rowperm != nullptr;
    std::vector<Field> fl = fields(d, has_perm);
    std::vector<int64_t> len(fl.size());
    size_t need = 16 + 16 + pad8(sizeof(BlobScalars));
    for (size_t i = 0; i < fl.size(); ++i) {
        len[i] = length_of(fl[i]);
        if (len[i] < 0) return err(H2B_ERR_INVALID, "h2b_map_blob_write: CSR array for field %u missing", fl[i].tag);
        if (len[i] > 0 && !*fl[i].ptr) return err(H2B_ERR_INVALID, "h2b_map_blob_write: field %u is NULL", fl[i].tag);
        need += 16 + pad8((size_t)len[i] * fl[i].elem);
    }
    *size = need;
    if (!buf) return H2B_OK;  // size query
    if (cap < need) return err(H2B_ERR_INVALID, "h2b_map_blob_write: buffer of %zu bytes, %zu needed", cap, need);
    BlobScalars sc{};
    sc.field = d.field;
    sc.precision = d.precision;
    sc.ncomp = d.ncomp;
    sc.dim = d.dim;
    sc.nsectors = d.nsectors;
    sc.transfer_kind = d.transfer_kind;
    sc.coupling_kind = d.coupling_kind;
    sc.conj_leaf_adjoint = d.conj_leaf_adjoint;
    std::memcpy(sc.alpha, d.alpha, sizeof(sc.alpha));
    sc.ncouplings = d.ncouplings;
    sc.coupling_len = d.coupling_len;
    sc.near_nrows = d.near_nrows;
    sc.near_kind = d.near_kind;
    sc.near_len = d.near_len;
    sc.near_wavenumber = d.near_wavenumber;
    sc.coupling_perm_len = d.coupling_perm_len;
    sc.has_perm = has_perm;
    for (int si = 0; si < 2; ++si) {
        const h2b_side_desc &s = si == 0 ? d.test : d.trial;
        sc.side[si] = {s.nnodes, s.nlevels, s.root, s.ndofs, s.agg_nstages, s.dis_nstages, s.coll_len, s.transfer_len};
    }
    unsigned char *o = static_cast<unsigned char *>(buf);
    std::memset(o, 0, need);
    std::memcpy(o, kMagic, 8);
    const uint64_t nrec = fl.size() + 1;
    std::memcpy(o + 8, &nrec, 8);
    size_t at = 16;
    auto put = [&](uint32_t tag, uint32_t elem, int64_t count, const void *src) {
        std::memcpy(o + at, &tag, 4);
        std::memcpy(o + at + 4, &elem, 4);
        std::memcpy(o + at + 8, &count, 8);
        at += 16;
        if (count > 0) std::memcpy(o + at, src, (size_t)count * elem);
        at += pad8((size_t)count * elem);
    };
    put(1, sizeof(BlobScalars), 1, &sc);
    for (size_t i = 0; i < fl.size(); ++i) put(fl[i].tag, fl[i].elem, len[i], *fl[i].ptr);
    return H2B_OK;
}

h2b_status h2b_map_blob_read(const void *blob, size_t bytes, h2b_map_desc *out) {
    if (!blob || !out) return err(H2B_ERR_INVALID, "h2b_map_blob_read: NULL argument");
    const unsigned char *b = static_cast<const unsigned char *>(blob);
    if ((reinterpret_cast<uintptr_t>(b) & 7) != 0)
        return err(H2B_ERR_INVALID, "h2b_map_blob_read: the blob must be 8-byte aligned");
    if (bytes < 32 + sizeof(BlobScalars) || std::memcmp(b, kMagic, 8) != 0)
        return err(H2B_ERR_INVALID, "h2b_map_blob_read: not a map blob");
    uint64_t nrec;
    std::memcpy(&nrec, b + 8, 8);
    size_t at = 16;
    // next record header, bounds-checked against the buffer
    auto next = [&](uint32_t &tag, uint32_t &elem, int64_t &count, const unsigned char *&data) -> bool {
        if (at + 16 > bytes) return false;
        std::memcpy(&tag, b + at, 4);
        std::memcpy(&elem, b + at + 4, 4);
        std::memcpy(&count, b + at + 8, 8);
        at += 16;
        if (count < 0 || elem == 0 || elem > 4096 || (uint64_t)count > (bytes - at) / elem) return false;
        data = b + at;
        at += pad8((size_t)count * elem);
        return at <= bytes;
    };
    uint32_t tag, elem;
    int64_t count;
    const unsigned char *data;
    if (nrec < 1 || !next(tag, elem, count, data) || tag != 1 || elem != sizeof(BlobScalars) || count != 1)
        return err(H2B_ERR_INVALID, "h2b_map_blob_read: missing scalars");
    BlobScalars sc;
    std::memcpy(&sc, data, sizeof(sc));
    h2b_map_desc d{};
    d.field = sc.field;
    d.precision = sc.precision;
    d.ncomp = sc.ncomp;
    d.dim = sc.dim;
    d.nsectors = sc.nsectors;
    d.transfer_kind = sc.transfer_kind;
    d.coupling_kind = sc.coupling_kind;
    d.conj_leaf_adjoint = sc.conj_leaf_adjoint;
    std::memcpy(d.alpha, sc.alpha, sizeof(d.alpha));
    d.ncouplings = sc.ncouplings;
    d.coupling_len = sc.coupling_len;
    d.near_nrows = sc.near_nrows;
    d.near_kind = sc.near_kind;
    d.near_len = sc.near_len;
    d.near_wavenumber = sc.near_wavenumber;
    d.coupling_perm_len = sc.coupling_perm_len;
    for (int si = 0; si < 2; ++si) {
        h2b_side_desc &s = si == 0 ? d.test : d.trial;
        const BlobSide &bs = sc.side[si];
        s.nnodes = bs.nnodes;
        s.nlevels = bs.nlevels;
        s.root = bs.root;
        s.ndofs = bs.ndofs;
        s.agg_nstages = bs.agg_nstages;
        s.dis_nstages = bs.dis_nstages;
        s.coll_len = bs.coll_len;
        s.transfer_len = bs.transfer_len;
    }
    if (d.test.nnodes < 1 || d.trial.nnodes < 1 || d.test.nlevels < 1 || d.trial.nlevels < 1 || d.nsectors < 1 ||
        d.nsectors > 8 || d.ncouplings < 0 || d.near_nrows < 0 || d.test.agg_nstages < 0 || d.trial.agg_nstages < 0 ||
        d.test.dis_nstages < 0 || d.trial.dis_nstages < 0)
        return err(H2B_ERR_INVALID, "h2b_map_blob_read: bad sizes");
    std::vector<Field> fl = fields(d, sc.has_perm != 0);
    if (nrec != fl.size() + 1)
        return err(H2B_ERR_INVALID, "h2b_map_blob_read: %llu records, %zu expected", (unsigned long long)nrec, fl.size() + 1);
    for (const Field &f : fl) {
        if (!next(tag, elem, count, data)) return err(H2B_ERR_INVALID, "h2b_map_blob_read: truncated blob");
        if (tag != f.tag || elem != f.elem)
            return err(H2B_ERR_INVALID, "h2b_map_blob_read: record for field %u where %u belongs", tag, f.tag);
        const int64_t want = length_of(f);  // CSR arrays this depends on are already set
        if (want < 0 || count != want)
            return err(H2B_ERR_INVALID, "h2b_map_blob_read: field %u has %lld entries, %lld expected", f.tag,
                       (long long)count, (long long)want);
        *f.ptr = data;
    }
    *out = d;
    return H2B_OK;
}

h2b_status h2b_core_create_from_blob(const void *blob, size_t bytes, int32_t device, h2b_core **out) {
    h2b_map_desc d;
    const h2b_status st = h2b_map_blob_read(blob, bytes, &d);
    if (st) return st;
    return h2b_core_create(&d, device, out);
}

}  // extern "C"
