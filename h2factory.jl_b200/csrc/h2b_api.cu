// C ABI of the B200 H2 matvec: core upload and validation, workspaces, and the orchestration of
// the near and far passes (LinearMaps._unsafe_mul! on an H2 map, src/maps/abstracth2map.jl:42-86).
//
// Every index array of the descriptor is validated on the host before anything reaches the GPU,
// so no kernel can be handed an out-of-range node, dof, coupling or block offset.

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "h2b_internal.cuh"

using namespace h2b;

namespace {

thread_local std::string g_err;

h2b_status fail(h2b_status st, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return st;
}

}  // namespace

h2b_status h2b::set_error_text(h2b_status st, const char *msg) {
    g_err = msg;
    return st;
}

namespace {

#define CUDA_TRY(expr)                                                                         \
    do {                                                                                       \
        cudaError_t e_ = (expr);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(e_ == cudaErrorMemoryAllocation ? H2B_ERR_NOMEM : H2B_ERR_CUDA,        \
                        "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

struct Stage {
    int level = 0;
    int n = 0;
    int *d_nodes = nullptr;
};

struct SideHost {
    int nnodes = 0, nlevels = 0, ndofs = 0;
    std::vector<int> level, shape;
    int maxcoef = 1, maxtsize = 1, maxvals = 1;
    int maxsep = 1;  // bound on separable-contraction intermediates between adjacent levels
    int maxaxis = 1; // longest padded Toeplitz axis (2s - 1)
    int64_t mom_total = 0, spec_total = 0;  // per unit right-hand side
    int *d_agg_leaves = nullptr;
    int n_agg_leaves = 0;
    std::vector<Stage> agg_inner;           // bottom-up
    int *d_store = nullptr;
    int n_store = 0;
    int *d_recv = nullptr;
    int n_recv = 0;
    std::vector<Stage> dis_down;            // top-down, nodes with a disaggregation parent
    uint8_t *d_received = nullptr;
    int *d_init_leaves = nullptr;
    int n_init_leaves = 0;
    int64_t npairs = 0;
    SibGroups sib;                      // Toeplitz I2O by sibling groups (ngroups = 0: per node)
    GroupTiles grp;                     // dense I2O for few right-hand sides, grouped by stored block
    int maxslen = 1;
    std::vector<int64_t> mom_off_host;  // moment offsets per unit rhs (host copy)
    std::vector<int64_t> spec_off_host; // spectrum offsets per unit rhs (host copy)
    int maxhalf = 1;                    // longest stored (half) spectrum
    DSide d{};
};

}  // namespace

struct h2b_core {
    int device = 0;
    int field = H2B_REAL, precision = H2B_FP64;
    bool conj_leaf = false;
    cdouble alpha[3];
    DMap dmap{};
    DNear dnear{};
    SideHost test, trial;
    int64_t near_entries = 0;
    std::vector<void *> allocs;
    int64_t bytes = 0;

    template <class X>
    cudaError_t alloc(X **p, size_t count) {
        *p = nullptr;
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc((void **)p, count * sizeof(X));
        if (e == cudaSuccess) {
            allocs.push_back((void *)*p);
            bytes += (int64_t)(count * sizeof(X));
        }
        return e;
    }
    template <class X>
    cudaError_t upload(X **p, const X *src, size_t count) {
        cudaError_t e = alloc(p, count);
        if (e != cudaSuccess || count == 0) return e;
        return cudaMemcpy(*p, src, count * sizeof(X), cudaMemcpyHostToDevice);
    }
    void release() {
        for (void *p : allocs) cudaFree(p);
        allocs.clear();
    }
};

struct h2b_workspace {
    h2b_core *core = nullptr;
    int max_nrhs = 1;
    void *am = nullptr, *dm = nullptr, *as = nullptr, *ds = nullptr;
    void *xbuf = nullptr, *ybuf = nullptr;  // staging for h2b_matvec_host
    void *xnear = nullptr;  // gathered x rows for the tensor-core near kernel (real, >= 8 RHS)
    unsigned *timeouts = nullptr;  // pinned: the device's tensor-core wait timeouts before / after a call
    std::atomic<int> busy{0};
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_done = nullptr, ev_far = nullptr;
    std::vector<void *> allocs;
};

namespace {

// ---------------------------------------------------------------------------------------------
// Descriptor validation
// ---------------------------------------------------------------------------------------------
int64_t ncoef_host(const h2b_side_desc &s, int lvl) {
    return (int64_t)s.shape[3 * lvl] * s.shape[3 * lvl + 1] * s.shape[3 * lvl + 2];
}
int64_t tsize_host(const h2b_side_desc &s, int lvl) {
    return (2 * (int64_t)s.shape[3 * lvl] - 1) * (2 * (int64_t)s.shape[3 * lvl + 1] - 1) *
           (2 * (int64_t)s.shape[3 * lvl + 2] - 1);
}
bool isleaf(const h2b_side_desc &s, int n) { return s.child_ptr[n + 1] == s.child_ptr[n]; }
// stored spectrum length: the whole padded array, or its first-axis half for Hermitian spectra
int64_t spec_len(const h2b_side_desc &s, int lvl, bool half) {
    const int64_t t0 = 2 * (int64_t)s.shape[3 * lvl] - 1;
    return half ? (t0 / 2 + 1) * (tsize_host(s, lvl) / t0) : tsize_host(s, lvl);
}

h2b_status validate_side(const h2b_map_desc &d, const h2b_side_desc &s, const h2b_side_desc &other,
                         const char *name, std::vector<int64_t> &permlen) {
    if (s.nnodes < 1 || s.nlevels < 1 || s.ndofs < 0)
        return fail(H2B_ERR_INVALID, "%s: nnodes/nlevels must be positive", name);
    if (!s.level || !s.parent || !s.sector || !s.child_ptr || !s.value_ptr || !s.shape ||
        !s.agg_ptr || !s.dis_ptr || !s.agg_store || !s.dis_isnode || !s.i2o_ptr || !s.coll_offset ||
        !s.transfer_offset)
        return fail(H2B_ERR_INVALID, "%s: missing array", name);
    if (s.root < 0 || s.root >= s.nnodes || s.parent[s.root] != -1)
        return fail(H2B_ERR_INVALID, "%s: bad root", name);
    for (int l = 1; l <= s.nlevels; ++l) {
        for (int k = 0; k < 3; ++k)
            if (s.shape[3 * l + k] < 1 || s.shape[3 * l + k] > 64)
                return fail(H2B_ERR_INVALID, "%s: moment extent out of range at level %d", name, l);
        if (ncoef_host(s, l) > 4096)
            return fail(H2B_ERR_UNSUPPORTED, "%s: more than 4096 coefficients at level %d", name, l);
        for (int k = d.dim; k < 3; ++k)
            if (s.shape[3 * l + k] != 1)
                return fail(H2B_ERR_INVALID, "%s: extent of unused axis %d must be 1", name, k + 1);
    }
    if (s.child_ptr[0] != 0) return fail(H2B_ERR_INVALID, "%s: child_ptr[0] != 0", name);
    if (s.value_ptr[0] != 0) return fail(H2B_ERR_INVALID, "%s: value_ptr[0] != 0", name);
    for (int n = 0; n < s.nnodes; ++n) {
        if (s.level[n] < 1 || s.level[n] > s.nlevels) return fail(H2B_ERR_INVALID, "%s: level of node %d", name, n);
        if (s.child_ptr[n + 1] < s.child_ptr[n]) return fail(H2B_ERR_INVALID, "%s: child_ptr not monotone", name);
        if (s.value_ptr[n + 1] < s.value_ptr[n]) return fail(H2B_ERR_INVALID, "%s: value_ptr not monotone", name);
        if (n != s.root) {
            const int p = s.parent[n];
            if (p < 0 || p >= s.nnodes) return fail(H2B_ERR_INVALID, "%s: parent of node %d", name, n);
            if (s.level[n] != s.level[p] + 1) return fail(H2B_ERR_INVALID, "%s: level of node %d vs parent", name, n);
            if (s.sector[n] < 0 || s.sector[n] >= d.nsectors)
                return fail(H2B_ERR_INVALID, "%s: sector of node %d", name, n);
        }
        if (!isleaf(s, n) && s.value_ptr[n + 1] != s.value_ptr[n])
            return fail(H2B_ERR_INVALID, "%s: inner node %d owns values", name, n);
    }
    const int nch = s.child_ptr[s.nnodes];
    if (nch > 0 && !s.child) return fail(H2B_ERR_INVALID, "%s: missing children", name);
    for (int n = 0; n < s.nnodes; ++n)
        for (int k = s.child_ptr[n]; k < s.child_ptr[n + 1]; ++k) {
            const int c = s.child[k];
            if (c < 0 || c >= s.nnodes || s.parent[c] != n)
                return fail(H2B_ERR_INVALID, "%s: child %d of node %d", name, c, n);
        }
    const int nval = s.value_ptr[s.nnodes];
    if (nval > 0 && !s.value) return fail(H2B_ERR_INVALID, "%s: missing values", name);
    if (nval > s.ndofs) return fail(H2B_ERR_INVALID, "%s: more dof ids than dofs", name);
    std::vector<uint8_t> owned(s.ndofs, 0);  // every dof belongs to one leaf at most
    for (int k = 0; k < nval; ++k) {
        if (s.value[k] < 0 || s.value[k] >= s.ndofs) return fail(H2B_ERR_INVALID, "%s: dof id out of range", name);
        if (owned[s.value[k]]++) return fail(H2B_ERR_INVALID, "%s: dof %d in two leaves", name, s.value[k]);
    }

    // aggregation plan
    std::vector<uint8_t> inagg(s.nnodes, 0);
    if (s.agg_nstages < 0 || s.agg_ptr[0] != 0) return fail(H2B_ERR_INVALID, "%s: agg_ptr", name);
    for (int st = 0; st < s.agg_nstages; ++st) {
        if (s.agg_ptr[st + 1] < s.agg_ptr[st]) return fail(H2B_ERR_INVALID, "%s: agg_ptr not monotone", name);
        if (st > 0 && s.agg_level[st] >= s.agg_level[st - 1])
            return fail(H2B_ERR_INVALID, "%s: aggregation stages must go bottom-up", name);
        for (int k = s.agg_ptr[st]; k < s.agg_ptr[st + 1]; ++k) {
            const int n = s.agg_node[k];
            if (n < 0 || n >= s.nnodes || s.level[n] != s.agg_level[st])
                return fail(H2B_ERR_INVALID, "%s: aggregation node %d", name, n);
            if (inagg[n]) return fail(H2B_ERR_INVALID, "%s: aggregation node %d listed twice", name, n);
            for (int q = s.child_ptr[n]; q < s.child_ptr[n + 1]; ++q)
                if (!inagg[s.child[q]])
                    return fail(H2B_ERR_INVALID, "%s: child %d of aggregation node %d is not aggregated first",
                                name, s.child[q], n);
            inagg[n] = 1;
        }
    }
    // disaggregation plan
    std::vector<uint8_t> indis(s.nnodes, 0);
    if (s.dis_nstages < 0 || s.dis_ptr[0] != 0) return fail(H2B_ERR_INVALID, "%s: dis_ptr", name);
    if (s.i2o_ptr[0] != 0) return fail(H2B_ERR_INVALID, "%s: i2o_ptr[0] != 0", name);
    for (int n = 0; n < s.nnodes; ++n)
        if (s.i2o_ptr[n + 1] < s.i2o_ptr[n]) return fail(H2B_ERR_INVALID, "%s: i2o_ptr not monotone", name);
    for (int st = 0; st < s.dis_nstages; ++st) {
        if (s.dis_ptr[st + 1] < s.dis_ptr[st]) return fail(H2B_ERR_INVALID, "%s: dis_ptr not monotone", name);
        if (st > 0 && s.dis_level[st] <= s.dis_level[st - 1])
            return fail(H2B_ERR_INVALID, "%s: disaggregation stages must go top-down", name);
        for (int k = s.dis_ptr[st]; k < s.dis_ptr[st + 1]; ++k) {
            const int n = s.dis_node[k];
            if (n < 0 || n >= s.nnodes || s.level[n] != s.dis_level[st] || !s.dis_isnode[n])
                return fail(H2B_ERR_INVALID, "%s: disaggregation node %d", name, n);
            if (indis[n]) return fail(H2B_ERR_INVALID, "%s: disaggregation node %d listed twice", name, n);
            const bool recv = s.i2o_ptr[n + 1] > s.i2o_ptr[n];
            const bool fromparent = n != s.root && s.dis_isnode[s.parent[n]];
            if (fromparent && !indis[s.parent[n]])
                return fail(H2B_ERR_INVALID, "%s: parent of %d is disaggregated later", name, n);
            if (!recv && !fromparent)
                return fail(H2B_ERR_INVALID, "%s: disaggregation node %d receives nothing", name, n);
            indis[n] = 1;
        }
    }
    for (int n = 0; n < s.nnodes; ++n) {
        if (s.dis_isnode[n] && !indis[n]) return fail(H2B_ERR_INVALID, "%s: node %d flagged but not scheduled", name, n);
        if (s.i2o_ptr[n + 1] > s.i2o_ptr[n] && !indis[n])
            return fail(H2B_ERR_INVALID, "%s: receiving node %d is not a disaggregation node", name, n);
    }
    const int npairs = s.i2o_ptr[s.nnodes];
    if (npairs > 0 && (!s.i2o_src || !s.i2o_coupling)) return fail(H2B_ERR_INVALID, "%s: missing pairs", name);
    for (int n = 0; n < s.nnodes; ++n)
        for (int p = s.i2o_ptr[n]; p < s.i2o_ptr[n + 1]; ++p) {
            const int src = s.i2o_src[p];
            if (src < 0 || src >= other.nnodes) return fail(H2B_ERR_INVALID, "%s: pair source out of range", name);
            if (!other.agg_store[src])
                return fail(H2B_ERR_INVALID, "%s: pair source %d is not a stored aggregation node", name, src);
            const int64_t key = s.i2o_coupling[p];
            if (key < 0 || key >= d.ncouplings) return fail(H2B_ERR_INVALID, "%s: coupling index out of range", name);
            const int64_t off = d.coupling_offset[key];
            int64_t need;
            const int64_t nr = ncoef_host(s, s.level[n]), nt = ncoef_host(other, other.level[src]);
            const int fw = d.field == H2B_COMPLEX ? 2 : 1;
            if (d.coupling_kind == H2B_COUPLING_DENSE) need = nr * nt * fw;
            else if (d.coupling_kind == H2B_COUPLING_DIAGONAL) {
                if (nr != nt) return fail(H2B_ERR_INVALID, "%s: diagonal coupling between different sizes", name);
                need = nr * fw;
            } else {
                for (int k = 0; k < 3; ++k)
                    if (s.shape[3 * s.level[n] + k] != other.shape[3 * other.level[src] + k])
                        return fail(H2B_ERR_INVALID, "%s: Toeplitz pair with different moment shapes", name);
                need = tsize_host(s, s.level[n]) * 2;
            }
            if (off < 0 || off + need > d.coupling_len)
                return fail(H2B_ERR_INVALID, "%s: coupling %lld exceeds the coupling array", name, (long long)key);
            if (d.coupling_rowperm) {
                // permuted couplings: square dense blocks (one grid permutation per side) or
                // Toeplitz tensors; the length each permutation must have
                int64_t len;
                if (d.coupling_kind == H2B_COUPLING_DENSE) {
                    if (nr != nt) return fail(H2B_ERR_INVALID, "%s: permuted coupling between different sizes", name);
                    len = nr;
                } else if (d.coupling_kind == H2B_COUPLING_TOEPLITZ) {
                    len = tsize_host(s, s.level[n]);
                } else {
                    return fail(H2B_ERR_UNSUPPORTED, "permuted diagonal couplings");
                }
                if (permlen[key] >= 0 && permlen[key] != len)
                    return fail(H2B_ERR_INVALID, "%s: coupling %lld used with two sizes", name, (long long)key);
                permlen[key] = len;
            }
        }
    // leaf collections of every leaf either plan touches
    const int fw = d.field == H2B_COMPLEX ? 2 : 1;
    (void)fw;
    for (int n = 0; n < s.nnodes; ++n) {
        if (!isleaf(s, n) || (!inagg[n] && !indis[n])) continue;
        const int64_t nv = s.value_ptr[n + 1] - s.value_ptr[n];
        const int64_t off = s.coll_offset[n];
        if (off < 0 || off + d.ncomp * ncoef_host(s, s.level[n]) * nv > s.coll_len)
            return fail(H2B_ERR_INVALID, "%s: leaf collection of node %d out of range", name, n);
    }
    // transfers of every edge either plan uses
    for (int n = 0; n < s.nnodes; ++n) {
        if (n == s.root) continue;
        const int p = s.parent[n];
        const bool used = (inagg[p] && inagg[n]) || (indis[n] && s.dis_isnode[p]);
        if (!used) continue;
        const int64_t off = s.transfer_offset[(int64_t)s.level[n] * d.nsectors + s.sector[n]];
        int64_t need;
        if (d.transfer_kind == H2B_TRANSFER_DENSE) need = ncoef_host(s, s.level[p]) * ncoef_host(s, s.level[n]);
        else {
            need = 0;
            for (int k = 0; k < d.dim; ++k)
                need += (int64_t)s.shape[3 * s.level[p] + k] * s.shape[3 * s.level[n] + k];
        }
        if (off < 0 || off + need > s.transfer_len)
            return fail(H2B_ERR_INVALID, "%s: transfer (level %d, sector %d) missing", name, s.level[n], s.sector[n]);
    }
    return H2B_OK;
}

h2b_status validate(const h2b_map_desc &d) {
    if (d.field != H2B_REAL && d.field != H2B_COMPLEX) return fail(H2B_ERR_INVALID, "field must be H2B_REAL or H2B_COMPLEX");
    if (d.precision != H2B_FP64 && d.precision != H2B_FP32) return fail(H2B_ERR_INVALID, "precision must be H2B_FP64 or H2B_FP32");
    if (d.ncomp < 1 || d.ncomp > 16) return fail(H2B_ERR_INVALID, "ncomp must be 1..16");
    if (d.dim < 1 || d.dim > 3) return fail(H2B_ERR_INVALID, "dim must be 1..3");
    if (d.nsectors < 1 || d.nsectors > 64) return fail(H2B_ERR_INVALID, "nsectors must be 1..64");
    if (d.transfer_kind != H2B_TRANSFER_DENSE && d.transfer_kind != H2B_TRANSFER_SEPARABLE)
        return fail(H2B_ERR_INVALID, "unknown transfer kind");
    if (d.coupling_kind < H2B_COUPLING_DENSE || d.coupling_kind > H2B_COUPLING_TOEPLITZ)
        return fail(H2B_ERR_INVALID, "unknown coupling kind");
    if (d.ncouplings < 0 || (d.ncouplings > 0 && (!d.coupling_offset || !d.coupling)))
        return fail(H2B_ERR_INVALID, "coupling arrays");
    if (d.field == H2B_REAL)
        for (int m = 0; m < 3; ++m)
            if (d.alpha[m][1] != 0.0) return fail(H2B_ERR_INVALID, "complex alpha on a real map");
    for (const h2b_side_desc *s : {&d.test, &d.trial}) {
        if (!s->agg_store || s->nnodes < 1) return fail(H2B_ERR_INVALID, "side without nodes or agg_store");
        if ((s->coll_len > 0 && !s->coll) || (s->transfer_len > 0 && !s->transfer) || s->coll_len < 0 ||
            s->transfer_len < 0)
            return fail(H2B_ERR_INVALID, "collection/transfer array missing");
    }
    if (d.coupling_len < 0 || (d.coupling_len > 0 && !d.coupling)) return fail(H2B_ERR_INVALID, "coupling array missing");
    if (d.near_len < 0 || (d.near_len > 0 && !d.near)) return fail(H2B_ERR_INVALID, "near array missing");
    std::vector<int64_t> permlen(std::max<int64_t>(d.ncouplings, 1), -1);
    if (d.coupling_rowperm && (!d.coupling_perm || d.coupling_perm_len < 0 ||
                               (d.coupling_kind == H2B_COUPLING_DENSE && !d.coupling_colperm)))
        return fail(H2B_ERR_INVALID, "coupling permutation arrays");
    h2b_status st = validate_side(d, d.test, d.trial, "test", permlen);
    if (st) return st;
    st = validate_side(d, d.trial, d.test, "trial", permlen);
    if (st) return st;
    if (d.coupling_rowperm) {
        // every permutation within the array and a permutation of 0 .. len-1
        std::vector<int> seen;
        for (int64_t k = 0; k < d.ncouplings; ++k) {
            if (permlen[k] < 0) continue;
            for (int w = 0; w < 2; ++w) {
                const int64_t *po = w == 0 ? d.coupling_rowperm : d.coupling_colperm;
                if (!po || (w == 1 && d.coupling_kind != H2B_COUPLING_DENSE)) continue;
                const int64_t o = po[k];
                if (o < -1 || (o >= 0 && o + permlen[k] > d.coupling_perm_len))
                    return fail(H2B_ERR_INVALID, "coupling %lld: permutation out of range", (long long)k);
                if (o < 0) continue;
                seen.assign(permlen[k], 0);
                for (int64_t i = 0; i < permlen[k]; ++i) {
                    const int v = d.coupling_perm[o + i];
                    if (v < 0 || v >= permlen[k] || seen[v]++)
                        return fail(H2B_ERR_INVALID, "coupling %lld: not a permutation", (long long)k);
                }
            }
        }
    }
    if (d.coupling_kind == H2B_COUPLING_TOEPLITZ) {
        for (const h2b_side_desc *s : {&d.test, &d.trial})
            for (int l = 1; l <= s->nlevels; ++l)
                for (int k = 0; k < 3; ++k)
                    if (s->shape[3 * l + k] > 8)
                        return fail(H2B_ERR_UNSUPPORTED, "Toeplitz moments are limited to 8 points per axis");
    }
    // near blocks
    const bool stored = d.near_kind == H2B_NEAR_STORED;
    if (d.near_kind < H2B_NEAR_STORED || d.near_kind > H2B_NEAR_HELMHOLTZ)
        return fail(H2B_ERR_INVALID, "unknown near kind %d", d.near_kind);
    if (!stored && (!d.test_points || !d.trial_points))
        return fail(H2B_ERR_INVALID, "matrix-free near field without points");
    if (d.near_kind == H2B_NEAR_HELMHOLTZ && d.field != H2B_COMPLEX)
        return fail(H2B_ERR_INVALID, "Helmholtz near kernel on a real map");
    if (!stored && !std::isfinite(d.near_wavenumber)) return fail(H2B_ERR_INVALID, "near wavenumber");
    if (d.near_nrows < 0) return fail(H2B_ERR_INVALID, "near_nrows");
    if (d.near_nrows > 0 && (!d.near_row || !d.near_ptr || (stored && (!d.near_offset || !d.near))))
        return fail(H2B_ERR_INVALID, "near arrays");
    if (d.near_nrows > 0 && d.near_ptr[0] != 0) return fail(H2B_ERR_INVALID, "near_ptr[0] != 0");
    for (int g = 0; g < d.near_nrows; ++g) {
        const int row = d.near_row[g];
        if (row < 0 || row >= d.test.nnodes || !isleaf(d.test, row))
            return fail(H2B_ERR_INVALID, "near row group %d is not a test leaf", g);
        if (d.near_ptr[g + 1] < d.near_ptr[g]) return fail(H2B_ERR_INVALID, "near_ptr not monotone");
        const int64_t nr = d.test.value_ptr[row + 1] - d.test.value_ptr[row];
        for (int b = d.near_ptr[g]; b < d.near_ptr[g + 1]; ++b) {
            const int col = d.near_col[b];
            if (col < 0 || col >= d.trial.nnodes || !isleaf(d.trial, col))
                return fail(H2B_ERR_INVALID, "near block %d: column is not a trial leaf", b);
            const int64_t nc = d.trial.value_ptr[col + 1] - d.trial.value_ptr[col];
            if (stored && (d.near_offset[b] < 0 || d.near_offset[b] + nr * nc > d.near_len))
                return fail(H2B_ERR_INVALID, "near block %d exceeds the near array", b);
        }
    }
    return H2B_OK;
}

// ---------------------------------------------------------------------------------------------
// Upload
// ---------------------------------------------------------------------------------------------
template <class T>
void convert_scalars(const double *src, int64_t count_scalars, bool cplx, std::vector<T> &out);

template <>
void convert_scalars<double>(const double *src, int64_t n, bool, std::vector<double> &out) {
    out.assign(src, src + n);
}
template <>
void convert_scalars<float>(const double *src, int64_t n, bool, std::vector<float> &out) {
    out.resize(n);
    for (int64_t i = 0; i < n; ++i) out[i] = (float)src[i];
}
template <>
void convert_scalars<cdouble>(const double *src, int64_t n, bool, std::vector<cdouble> &out) {
    out.resize(n);
    for (int64_t i = 0; i < n; ++i) out[i] = {src[2 * i], src[2 * i + 1]};
}
template <>
void convert_scalars<cfloat>(const double *src, int64_t n, bool, std::vector<cfloat> &out) {
    out.resize(n);
    for (int64_t i = 0; i < n; ++i) out[i] = {(float)src[2 * i], (float)src[2 * i + 1]};
}

template <class T>
h2b_status upload_scalars(h2b_core *c, const double *src, int64_t count, const void **dst) {
    std::vector<T> tmp;
    convert_scalars<T>(src, count, ScalarTraits<T>::is_complex, tmp);
    T *p = nullptr;
    CUDA_TRY(c->upload(&p, tmp.data(), tmp.size()));
    *dst = p;
    return H2B_OK;
}

h2b_status upload_far_scalars(h2b_core *c, const double *src, int64_t count, const void **dst) {
    const bool cplx = c->field == H2B_COMPLEX;
    if (!cplx && c->precision == H2B_FP64) return upload_scalars<double>(c, src, count, dst);
    if (!cplx) return upload_scalars<float>(c, src, count, dst);
    if (c->precision == H2B_FP64) return upload_scalars<cdouble>(c, src, count, dst);
    return upload_scalars<cfloat>(c, src, count, dst);
}

h2b_status upload_list(h2b_core *c, const std::vector<int> &v, int **dst) {
    CUDA_TRY(c->upload(dst, v.data(), v.size()));
    return H2B_OK;
}

// Chunks and tiles of the grouped dense I2O (GroupTiles) for the receiving nodes of side `s`:
// chunks of up to GT_R consecutive receiving nodes of one level -- fewer when the map has too few
// receiving nodes to give every SM a full chunk (down to 4 per chunk: a small map trades block
// reuse for SMs; with two chunks per SM as the target the large maps lost more reuse than they
// gained SMs); per chunk, its pairs sorted by
// stored block, then by their rank among the receiver's pairs reading that block, then by receiver,
// and cut into tiles of at most GT_P pairs with one block and distinct receivers.
h2b_status build_group_tiles(h2b_core *c, const h2b_side_desc &s, SideHost &h,
                             const std::vector<int64_t> &cpl_elem_off) {
    std::vector<int> recv;
    for (int n = 0; n < s.nnodes; ++n)
        if (s.i2o_ptr[n + 1] > s.i2o_ptr[n]) recv.push_back(n);
    if (recv.empty()) return H2B_OK;
    int nsm = 148;
    CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    const int R = std::min(GT_R, std::max(4, (int)(recv.size() / (size_t)nsm)));
    std::vector<int> chunk_ptr{0}, rcv, tile_ptr{0}, tile_pp{0}, pair;
    std::vector<unsigned char> slot;
    struct E { int64_t key; int rank, slot, p; };
    size_t i = 0;
    while (i < recv.size()) {
        const int lvl = s.level[recv[i]];
        const size_t j0 = i;
        while (i < recv.size() && (int)(i - j0) < R && s.level[recv[i]] == lvl) rcv.push_back(recv[i++]);
        std::vector<E> es;
        for (size_t j = j0; j < i; ++j) {
            const int n = recv[j];
            std::map<int64_t, int> rank;
            for (int p = s.i2o_ptr[n]; p < s.i2o_ptr[n + 1]; ++p) {
                const int64_t key = cpl_elem_off[p];
                es.push_back({key, rank[key]++, (int)(j - j0), p});
            }
        }
        std::sort(es.begin(), es.end(), [](const E &a, const E &b) {
            return a.key != b.key ? a.key < b.key : (a.rank != b.rank ? a.rank < b.rank : a.slot < b.slot);
        });
        unsigned used = 0;
        int64_t key = -1;
        int len = 0;
        for (const E &e : es) {
            if (len > 0 && (e.key != key || len == GT_P || (used >> e.slot & 1u))) {
                tile_pp.push_back((int)pair.size());
                used = 0;
                len = 0;
            }
            key = e.key;
            used |= 1u << e.slot;
            ++len;
            pair.push_back(e.p);
            slot.push_back((unsigned char)e.slot);
        }
        if (len > 0) tile_pp.push_back((int)pair.size());
        chunk_ptr.push_back((int)rcv.size());
        tile_ptr.push_back((int)tile_pp.size() - 1);
    }
    GroupTiles &g = h.grp;
    int *q;
    unsigned char *u;
    CUDA_TRY(c->upload(&q, chunk_ptr.data(), chunk_ptr.size())); g.chunk_ptr = q;
    CUDA_TRY(c->upload(&q, rcv.data(), rcv.size())); g.rcv = q;
    CUDA_TRY(c->upload(&q, tile_ptr.data(), tile_ptr.size())); g.tile_ptr = q;
    CUDA_TRY(c->upload(&q, tile_pp.data(), tile_pp.size())); g.tile_pp = q;
    CUDA_TRY(c->upload(&q, pair.data(), pair.size())); g.pair = q;
    CUDA_TRY(c->upload(&u, slot.data(), slot.size())); g.slot = u;
    g.nchunks = (int)chunk_ptr.size() - 1;
    return H2B_OK;
}

// Sibling groups of the receiving nodes of side `s` for the Toeplitz I2O: the receiving children
// of each parent, with the union of their sources and, per (source, child slot), the coupling's
// element offset. Left empty (per-node kernel) when a receiver has no parent or a child slot
// beyond 8, or lists one source twice.
h2b_status build_sibling_groups(h2b_core *c, const h2b_side_desc &s, SideHost &h,
                                const std::vector<int64_t> &other_spec_off,
                                const std::vector<int64_t> &cpl_elem_off) {
    std::vector<int> recv;
    for (int n = 0; n < s.nnodes; ++n)
        if (s.i2o_ptr[n + 1] > s.i2o_ptr[n]) recv.push_back(n);
    std::map<int, int> gidx;
    std::vector<int> grecv;
    for (int n : recv) {
        if (n == s.root || s.sector[n] >= 8) return H2B_OK;
        auto it = gidx.find(s.parent[n]);
        if (it == gidx.end()) {
            it = gidx.emplace(s.parent[n], (int)gidx.size()).first;
            grecv.insert(grecv.end(), 8, -1);
        }
        grecv[it->second * 8 + s.sector[n]] = n;
    }
    const int ng = (int)gidx.size();
    std::vector<int> gptr{0}, gslen(ng), gkof;
    std::vector<int64_t> gsrc;
    for (int gi = 0; gi < ng; ++gi) {
        std::map<int, std::vector<int>> bysrc;
        for (int sl = 0; sl < 8; ++sl) {
            const int n = grecv[gi * 8 + sl];
            if (n < 0) continue;
            gslen[gi] = (int)spec_len(s, s.level[n], c->dmap.half_spectrum != 0);
            for (int p = s.i2o_ptr[n]; p < s.i2o_ptr[n + 1]; ++p) {
                auto &row = bysrc[s.i2o_src[p]];
                if (row.empty()) row.assign(8, -1);
                if (row[sl] >= 0) return H2B_OK;  // duplicate pair: keep the per-node kernel
                const int64_t ko = cpl_elem_off[s.i2o_coupling[p]];
                if (ko > INT32_MAX - 8192) return H2B_OK;  // offsets must fit 32 bits here
                row[sl] = (int)ko;
            }
        }
        if (gslen[gi] > 512) return H2B_OK;  // one thread per stored frequency: per-node kernel
        for (auto &kv : bysrc) {
            gsrc.push_back(other_spec_off[kv.first]);
            gkof.insert(gkof.end(), kv.second.begin(), kv.second.end());
        }
        gptr.push_back((int)gsrc.size());
    }
    SibGroups &g = h.sib;
    int *p;
    int64_t *q;
    CUDA_TRY(c->upload(&p, grecv.data(), std::max<size_t>(grecv.size(), 1))); g.recv = p;
    CUDA_TRY(c->upload(&p, gslen.data(), std::max<size_t>(gslen.size(), 1))); g.slen = p;
    CUDA_TRY(c->upload(&p, gptr.data(), gptr.size())); g.ptr = p;
    CUDA_TRY(c->upload(&q, gsrc.data(), std::max<size_t>(gsrc.size(), 1))); g.src_off = q;
    CUDA_TRY(c->upload(&p, gkof.data(), std::max<size_t>(gkof.size(), 1))); g.kof = p;
    g.ngroups = ng;
    for (int v : gslen) h.maxslen = std::max(h.maxslen, v);
    return H2B_OK;
}

h2b_status build_side(h2b_core *c, const h2b_map_desc &d, const h2b_side_desc &s, const h2b_side_desc &other,
                      SideHost &h) {
    h.nnodes = s.nnodes;
    h.nlevels = s.nlevels;
    h.ndofs = s.ndofs;
    h.level.assign(s.level, s.level + s.nnodes);
    h.shape.assign(s.shape, s.shape + 3 * (s.nlevels + 1));
    for (int l = 1; l <= s.nlevels; ++l) {
        h.maxcoef = std::max<int>(h.maxcoef, (int)ncoef_host(s, l));
        h.maxtsize = std::max<int>(h.maxtsize, (int)tsize_host(s, l));
        for (int k = 0; k < 3; ++k) h.maxaxis = std::max(h.maxaxis, 2 * s.shape[3 * l + k] - 1);
        if (l > 1) {
            int b = 1;
            for (int k = 0; k < 3; ++k) b *= std::max(s.shape[3 * l + k], s.shape[3 * (l - 1) + k]);
            h.maxsep = std::max(h.maxsep, b);
        }
    }
    for (int n = 0; n < s.nnodes; ++n) h.maxvals = std::max(h.maxvals, s.value_ptr[n + 1] - s.value_ptr[n]);
    DSide &D = h.d;
    D.nnodes = s.nnodes;
    D.nlevels = s.nlevels;
    D.ndofs = s.ndofs;
    D.nvalues = s.value_ptr[s.nnodes];
    int *p;
    CUDA_TRY(c->upload(&p, s.level, s.nnodes)); D.level = p;
    CUDA_TRY(c->upload(&p, s.parent, s.nnodes)); D.parent = p;
    CUDA_TRY(c->upload(&p, s.sector, s.nnodes)); D.sector = p;
    CUDA_TRY(c->upload(&p, s.child_ptr, s.nnodes + 1)); D.child_ptr = p;
    CUDA_TRY(c->upload(&p, s.child, s.child_ptr[s.nnodes])); D.child = p;
    CUDA_TRY(c->upload(&p, s.value_ptr, s.nnodes + 1)); D.value_ptr = p;
    CUDA_TRY(c->upload(&p, s.value, s.value_ptr[s.nnodes])); D.value = p;
    CUDA_TRY(c->upload(&p, s.shape, 3 * (s.nlevels + 1))); D.shape = p;
    CUDA_TRY(c->upload(&p, s.i2o_ptr, s.nnodes + 1)); D.i2o_ptr = p;
    CUDA_TRY(c->upload(&p, s.i2o_src, s.i2o_ptr[s.nnodes])); D.i2o_src = p;
    int64_t *q;
    CUDA_TRY(c->upload(&q, s.i2o_coupling, s.i2o_ptr[s.nnodes])); D.i2o_cpl = q;
    h.npairs = s.i2o_ptr[s.nnodes];

    // moment / spectrum slots per unit right-hand side
    std::vector<int64_t> mo(s.nnodes), so(s.nnodes);
    int64_t mt = 0, stot = 0;
    const bool toep = d.coupling_kind == H2B_COUPLING_TOEPLITZ;
    for (int n = 0; n < s.nnodes; ++n) {
        mo[n] = mt;
        so[n] = stot;
        mt += d.ncomp * ncoef_host(s, s.level[n]);
        if (toep) stot += d.ncomp * spec_len(s, s.level[n], c->dmap.half_spectrum != 0);
    }
    h.mom_total = mt;
    h.spec_total = stot;
    CUDA_TRY(c->upload(&q, mo.data(), mo.size())); D.mom_off = q;
    CUDA_TRY(c->upload(&q, so.data(), so.size())); D.spec_off = q;

    // leaf collections and transfers in the far-field precision
    const int fw = d.field == H2B_COMPLEX ? 2 : 1;
    h2b_status st = upload_far_scalars(c, s.coll, s.coll_len, &D.coll);
    if (st) return st;
    CUDA_TRY(c->upload(&q, s.coll_offset, s.nnodes)); D.coll_off = q;
    st = upload_far_scalars(c, s.transfer, s.transfer_len, &D.tr);
    if (st) return st;
    CUDA_TRY(c->upload(&q, s.transfer_offset, (size_t)(s.nlevels + 1) * d.nsectors)); D.tr_off = q;
    (void)fw;

    // node lists
    std::vector<int> leaves;
    for (int st2 = 0; st2 < s.agg_nstages; ++st2) {
        Stage sg;
        sg.level = s.agg_level[st2];
        std::vector<int> inner;
        for (int k = s.agg_ptr[st2]; k < s.agg_ptr[st2 + 1]; ++k) {
            const int n = s.agg_node[k];
            if (isleaf(s, n)) leaves.push_back(n);
            else inner.push_back(n);
        }
        sg.n = (int)inner.size();
        st = upload_list(c, inner, &sg.d_nodes);
        if (st) return st;
        h.agg_inner.push_back(sg);
    }
    h.n_agg_leaves = (int)leaves.size();
    st = upload_list(c, leaves, &h.d_agg_leaves);
    if (st) return st;
    std::vector<int> store;
    for (int n = 0; n < s.nnodes; ++n)
        if (s.agg_store[n]) store.push_back(n);
    h.n_store = (int)store.size();
    st = upload_list(c, store, &h.d_store);
    if (st) return st;

    std::vector<int> recv, initleaves;
    std::vector<uint8_t> received(s.nnodes, 0);
    for (int st2 = 0; st2 < s.dis_nstages; ++st2) {
        Stage sg;
        sg.level = s.dis_level[st2];
        std::vector<int> down;
        for (int k = s.dis_ptr[st2]; k < s.dis_ptr[st2 + 1]; ++k) {
            const int n = s.dis_node[k];
            const bool r = s.i2o_ptr[n + 1] > s.i2o_ptr[n];
            const bool fp = n != s.root && s.dis_isnode[s.parent[n]];
            if (r) { recv.push_back(n); received[n] = 1; }
            if (fp) down.push_back(n);
            if (isleaf(s, n) && (r || fp)) initleaves.push_back(n);
        }
        sg.n = (int)down.size();
        st = upload_list(c, down, &sg.d_nodes);
        if (st) return st;
        h.dis_down.push_back(sg);
    }
    h.n_recv = (int)recv.size();
    st = upload_list(c, recv, &h.d_recv);
    if (st) return st;
    h.n_init_leaves = (int)initleaves.size();
    st = upload_list(c, initleaves, &h.d_init_leaves);
    if (st) return st;
    CUDA_TRY(c->upload(&h.d_received, received.data(), received.size()));
    (void)other;
    h.mom_off_host = mo;
    h.spec_off_host = so;
    for (int l = 1; l <= s.nlevels; ++l)
        h.maxhalf = std::max<int>(h.maxhalf, (int)spec_len(s, l, c->dmap.half_spectrum != 0));
    return H2B_OK;
}

// Near blocks: repacked into the padded column-major layout of the near kernel (h2b_near.cu),
// grouped by output leaf. N^T is needed for transpose/adjoint products: when the test and trial
// sides are the same tree and every block equals the transpose of its mirror block (checked on the
// device), N^T == N and N serves both; otherwise a transposed copy is built once here.
h2b_status build_near(h2b_core *c, const h2b_map_desc &d) {
    const bool cplx = d.field == H2B_COMPLEX;
    const size_t vb = cplx ? 2 * sizeof(double) : sizeof(double);
    const int nb = d.near_nrows > 0 ? d.near_ptr[d.near_nrows] : 0;
    std::vector<int> blk_row(nb), blk_col(nb);
    std::vector<int64_t> src_off(nb), fwd_off(nb), tr_off(nb);
    int64_t entries = 0, fwd_len = 0, tr_len = 0;
    auto nv = [](const h2b_side_desc &s, int n) { return s.value_ptr[n + 1] - s.value_ptr[n]; };
    for (int g = 0; g < d.near_nrows; ++g)
        for (int b = d.near_ptr[g]; b < d.near_ptr[g + 1]; ++b) {
            blk_row[b] = d.near_row[g];
            blk_col[b] = d.near_col[b];
            src_off[b] = d.near_offset[b];
            const int nr = nv(d.test, blk_row[b]), nc = nv(d.trial, blk_col[b]);
            entries += (int64_t)nr * nc;
            fwd_off[b] = fwd_len;
            fwd_len += near_padded_ld(cplx, nr) * nc;
            tr_off[b] = tr_len;
            tr_len += near_padded_ld(cplx, nc) * nr;
        }
    c->near_entries = d.near_kind == H2B_NEAR_STORED ? entries : 0;
    // groups over every output leaf, so that leaves without near blocks still get y = beta * y
    auto groups = [&](const h2b_side_desc &s, const std::vector<int> &key, std::vector<int> &leaf,
                      std::vector<int> &ptr, std::vector<int> &blk) {
        std::vector<int> slot(s.nnodes, -1);
        for (int n = 0; n < s.nnodes; ++n)
            if (isleaf(s, n)) { slot[n] = (int)leaf.size(); leaf.push_back(n); }
        ptr.assign(leaf.size() + 1, 0);
        for (int b = 0; b < nb; ++b) ptr[slot[key[b]] + 1]++;
        for (size_t g = 0; g < leaf.size(); ++g) ptr[g + 1] += ptr[g];
        blk.assign(std::max(nb, 1), 0);
        std::vector<int> fill(ptr.begin(), ptr.end() - 1);
        for (int b = 0; b < nb; ++b) blk[fill[slot[key[b]]]++] = b;
    };
    // work units of every group in block order: {first input value, columns (<= 32), element
    // offset of the chunk's first column in the padded layout (low, high 32 bits)}
    auto units = [&](NearOp &op, const h2b_side_desc &out, const h2b_side_desc &in, const std::vector<int> &key_in,
                     const std::vector<int> &leaf, const std::vector<int> &ptr, const std::vector<int> &blk,
                     const std::vector<int64_t> &off) -> h2b_status {
        std::vector<int> uptr(leaf.size() + 1, 0);
        std::vector<int4> ulist;
        for (size_t g = 0; g < leaf.size(); ++g) {
            const int64_t ld = near_padded_ld(cplx, nv(out, leaf[g]));
            for (int bb = ptr[g]; bb < ptr[g + 1]; ++bb) {
                const int b = blk[bb], c0 = in.value_ptr[key_in[b]], nc = nv(in, key_in[b]);
                for (int j0 = 0; j0 < nc; j0 += 32) {
                    const int64_t o = off[b] + j0 * ld;
                    ulist.push_back(make_int4(c0 + j0, std::min(32, nc - j0), (int)(uint32_t)o, (int)(o >> 32)));
                }
            }
            uptr[g + 1] = (int)ulist.size();
        }
        if (ulist.empty()) ulist.push_back(make_int4(0, 0, 0, 0));
        std::vector<int2> slabs;
        for (size_t g = 0; g < leaf.size(); ++g)
            for (int r0 = 0; r0 < nv(out, leaf[g]); r0 += 32) slabs.push_back(make_int2((int)g, r0 / 32));
        op.nslabs = (int)slabs.size();
        if (slabs.empty()) slabs.push_back(make_int2(0, 0));
        int *pp;
        int4 *pu;
        int2 *ps;
        CUDA_TRY(c->upload(&pp, uptr.data(), uptr.size()));
        CUDA_TRY(c->upload(&pu, ulist.data(), ulist.size()));
        CUDA_TRY(c->upload(&ps, slabs.data(), slabs.size()));
        op.unit_ptr = pp;
        op.unit = pu;
        op.slab = ps;
        return H2B_OK;
    };
    int *p;
    int64_t *q;
    int *d_row, *d_col;
    int64_t *d_src_off;
    CUDA_TRY(c->upload(&d_row, blk_row.data(), blk_row.size()));
    CUDA_TRY(c->upload(&d_col, blk_col.data(), blk_col.size()));

    if (d.near_kind != H2B_NEAR_STORED) {
        // matrix-free: the block structure in both orientations, the points, no block data
        DNear &dn = c->dnear;
        dn.kind = d.near_kind;
        dn.wavenumber = d.near_wavenumber;
        double *pts;
        CUDA_TRY(c->upload(&pts, d.test_points, (size_t)3 * std::max(d.test.ndofs, 1)));
        dn.test_pts = pts;
        CUDA_TRY(c->upload(&pts, d.trial_points, (size_t)3 * std::max(d.trial.ndofs, 1)));
        dn.trial_pts = pts;
        for (int side = 0; side < 2; ++side) {
            std::vector<int> leaf, ptr, blk;
            groups(side == 0 ? d.test : d.trial, side == 0 ? blk_row : blk_col, leaf, ptr, blk);
            NearOp &op = side == 0 ? dn.fwd : dn.tr;
            CUDA_TRY(c->upload(&p, leaf.data(), leaf.size())); op.grp_leaf = p;
            op.ngroups = (int)leaf.size();
            if (h2b_status us = units(op, side == 0 ? d.test : d.trial, side == 0 ? d.trial : d.test,
                                      side == 0 ? blk_col : blk_row, leaf, ptr, blk, side == 0 ? fwd_off : tr_off))
                return us;
        }
        dn.symmetric = false;
        CUDA_TRY(cudaDeviceSynchronize());
        return H2B_OK;
    }
    CUDA_TRY(c->upload(&d_src_off, src_off.data(), src_off.size()));

    // source blocks on the device (the caller's device buffer, or a temporary upload)
    const void *src = d.near;
    void *tmp = nullptr;
    if (!d.near_on_device && d.near_len > 0) {
        CUDA_TRY(cudaMalloc(&tmp, (size_t)d.near_len * vb));
        cudaError_t e = cudaMemcpy(tmp, d.near, (size_t)d.near_len * vb, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(tmp);
            return fail(H2B_ERR_CUDA, "near upload failed: %s", cudaGetErrorString(e));
        }
        src = tmp;
    }
    struct TmpGuard {
        void *p;
        ~TmpGuard() { if (p) cudaFree(p); }
    } tguard{tmp};

    // N in the padded layout, grouped by test leaf
    {
        std::vector<int> leaf, ptr, blk;
        groups(d.test, blk_row, leaf, ptr, blk);
        NearOp &op = c->dnear.fwd;
        CUDA_TRY(c->upload(&p, leaf.data(), leaf.size())); op.grp_leaf = p;
        CUDA_TRY(c->upload(&q, fwd_off.data(), fwd_off.size())); op.blk_off = q;
        if (h2b_status us = units(op, d.test, d.trial, blk_col, leaf, ptr, blk, fwd_off)) return us;
        unsigned char *data;
        CUDA_TRY(c->alloc(&data, (size_t)std::max<int64_t>(fwd_len, 2) * vb));
        op.data = data;
        op.ngroups = (int)leaf.size();
        if (nb > 0)
            CUDA_TRY(launch_near_repack(cplx, src, d_src_off, d_row, d_col, c->test.d, c->trial.d, data,
                                        op.blk_off, nb, false, 0));
    }

    // N^T == N ?
    bool symmetric = false;
    const bool same_tree = d.test.nnodes == d.trial.nnodes && d.test.ndofs == d.trial.ndofs &&
                           std::equal(d.test.value_ptr, d.test.value_ptr + d.test.nnodes + 1, d.trial.value_ptr) &&
                           std::equal(d.test.value, d.test.value + d.test.value_ptr[d.test.nnodes], d.trial.value);
    if (same_tree) {
        std::vector<int> mirror(std::max(nb, 1), -1);
        std::vector<int64_t> key(nb);
        std::vector<int> order(nb);
        for (int b = 0; b < nb; ++b) {
            key[b] = (int64_t)blk_row[b] * d.test.nnodes + blk_col[b];
            order[b] = b;
        }
        std::sort(order.begin(), order.end(), [&](int a, int b2) { return key[a] < key[b2]; });
        bool all = true;
        for (int b = 0; b < nb && all; ++b) {
            const int64_t want = (int64_t)blk_col[b] * d.test.nnodes + blk_row[b];
            auto it = std::lower_bound(order.begin(), order.end(), want,
                                       [&](int a, int64_t v) { return key[a] < v; });
            if (it == order.end() || key[*it] != want) all = false;
            else mirror[b] = *it;
        }
        if (all) {
            int *d_mirror, *d_flag;
            CUDA_TRY(c->upload(&d_mirror, mirror.data(), mirror.size()));
            const int one = 1;
            CUDA_TRY(c->upload(&d_flag, &one, 1));
            CUDA_TRY(launch_near_symcheck(cplx, src, d_src_off, d_mirror, d_row, c->test.d, nb, d_flag, 0));
            int flag = 0;
            CUDA_TRY(cudaMemcpy(&flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost));
            symmetric = flag == 1;
        }
    }
    c->dnear.symmetric = symmetric;

    if (!symmetric) {
        // N^T in the padded layout, grouped by trial leaf
        std::vector<int> leaf, ptr, blk;
        groups(d.trial, blk_col, leaf, ptr, blk);
        NearOp &op = c->dnear.tr;
        CUDA_TRY(c->upload(&p, leaf.data(), leaf.size())); op.grp_leaf = p;
        CUDA_TRY(c->upload(&q, tr_off.data(), tr_off.size())); op.blk_off = q;
        if (h2b_status us = units(op, d.trial, d.test, blk_row, leaf, ptr, blk, tr_off)) return us;
        unsigned char *data;
        CUDA_TRY(c->alloc(&data, (size_t)std::max<int64_t>(tr_len, 2) * vb));
        op.data = data;
        op.ngroups = (int)leaf.size();
        if (nb > 0)
            CUDA_TRY(launch_near_repack(cplx, src, d_src_off, d_row, d_col, c->test.d, c->trial.d, data,
                                        op.blk_off, nb, true, 0));
    }
    CUDA_TRY(cudaDeviceSynchronize());
    return H2B_OK;
}

// The FP32 form's dense couplings transposed block by block (same offsets), for the tensor-core
// I2O's transposed and adjoint products, and whether every block is laid out for 16-byte bulk
// copies of its columns. A block's shape is (receiver coefficients x source coefficients) of the
// test-side pairs that use it.
h2b_status build_transposed_couplings(h2b_core *c, const h2b_map_desc &d, const std::vector<int64_t> &off) {
    const bool cplx = d.field == H2B_COMPLEX;
    const int fw = cplx ? 2 : 1;
    const int64_t n = d.coupling_len / fw;  // elements
    std::vector<int64_t> rows(std::max<int64_t>(d.ncouplings, 1), -1), cols(rows.size(), -1);
    for (int r = 0; r < d.test.nnodes; ++r)
        for (int p = d.test.i2o_ptr[r]; p < d.test.i2o_ptr[r + 1]; ++p) {
            const int64_t k = d.test.i2o_coupling[p];
            rows[k] = ncoef_host(d.test, d.test.level[r]);
            cols[k] = ncoef_host(d.trial, d.trial.level[d.test.i2o_src[p]]);
        }
    std::vector<double> tr((size_t)std::max<int64_t>(n, 1) * fw, 0.0);
    const int eb = 4 * fw;  // bytes per FP32 element
    bool vec = true;
    std::vector<char> done((size_t)std::max<int64_t>(n, 1), 0);
    for (int64_t k = 0; k < d.ncouplings; ++k) {
        if (rows[k] < 0) continue;
        const int64_t o = off[k], nr = rows[k], nc = cols[k];
        vec &= (o * eb) % 16 == 0 && (nr * eb) % 16 == 0 && (nc * eb) % 16 == 0;
        if (done[o]) continue;  // symmetry-reduced couplings share their canonical block
        done[o] = 1;
        for (int64_t j = 0; j < nc; ++j)
            for (int64_t i = 0; i < nr; ++i)
                for (int w = 0; w < fw; ++w)
                    tr[(size_t)(o + j + i * nc) * fw + w] = d.coupling[(size_t)(o + i + j * nr) * fw + w];
    }
    c->dmap.cpl_vec = vec ? 1 : 0;
    return upload_far_scalars(c, tr.data(), std::max<int64_t>(n, 1), &c->dmap.cpl_t);
}

// Padded shape (2s - 1 per axis) of every coupling, from the pairs that use it; 0 if unused.
std::vector<int> coupling_shapes(const h2b_map_desc &d) {
    std::vector<int> ts(3 * std::max<int64_t>(d.ncouplings, 1), 0);
    for (const h2b_side_desc *s : {&d.test, &d.trial})
        for (int n = 0; n < s->nnodes; ++n)
            for (int p = s->i2o_ptr[n]; p < s->i2o_ptr[n + 1]; ++p)
                for (int k = 0; k < 3; ++k) ts[3 * s->i2o_coupling[p] + k] = 2 * s->shape[3 * s->level[n] + k] - 1;
    return ts;
}

// Is every used Toeplitz coupling Hermitian, K[k] == conj(K[-k]) to rounding?
bool couplings_hermitian(const h2b_map_desc &d, const std::vector<int> &ts) {
    for (int64_t c = 0; c < d.ncouplings; ++c) {
        const int n0 = ts[3 * c], n1 = ts[3 * c + 1], n2 = ts[3 * c + 2];
        if (n0 == 0) continue;
        const double *K = d.coupling + d.coupling_offset[c];
        double mx = 0.0;
        for (int64_t e = 0; e < (int64_t)n0 * n1 * n2; ++e) mx = std::max(mx, std::hypot(K[2 * e], K[2 * e + 1]));
        const double tol = 1e-12 * std::max(mx, 1e-300);
        for (int k3 = 0; k3 < n2; ++k3)
            for (int k2 = 0; k2 < n1; ++k2)
                for (int k1 = 0; k1 < n0; ++k1) {
                    const int64_t e = k1 + (int64_t)n0 * (k2 + (int64_t)n1 * k3);
                    const int64_t f = (n0 - k1) % n0 + (int64_t)n0 * ((n1 - k2) % n1 + (int64_t)n1 * ((n2 - k3) % n2));
                    if (std::fabs(K[2 * e] - K[2 * f]) > tol || std::fabs(K[2 * e + 1] + K[2 * f + 1]) > tol)
                        return false;
                }
    }
    return true;
}

h2b_status build_core(h2b_core *c, const h2b_map_desc &d) {
    DMap &M = c->dmap;
    M.ncomp = d.ncomp;
    M.dim = d.dim;
    M.nsectors = d.nsectors;
    M.transfer_kind = d.transfer_kind;
    M.coupling_kind = d.coupling_kind;
    const bool cplx = d.field == H2B_COMPLEX;
    const bool toep = d.coupling_kind == H2B_COUPLING_TOEPLITZ;
    std::vector<int> ts;
    if (toep) ts = coupling_shapes(d);
    M.half_spectrum = toep && !cplx && couplings_hermitian(d, ts);
    // specialised transforms when every level of both sides has (p, p, p) moments with 2p - 1 == 7
    M.cube_ts = 0;
    if (toep && d.dim == 3) {
        bool cube = true;
        for (const h2b_side_desc *sd : {&d.test, &d.trial})
            for (int l = 1; l <= sd->nlevels; ++l)
                cube &= sd->shape[3 * l] == 4 && sd->shape[3 * l + 1] == 4 && sd->shape[3 * l + 2] == 4;
        if (cube) M.cube_ts = 7;
    }
    h2b_status st = build_side(c, d, d.test, d.trial, c->test);
    if (st) return st;
    st = build_side(c, d, d.trial, d.test, c->trial);
    if (st) return st;
    // coupling data: offsets arrive in doubles; convert to elements of the device type
    std::vector<int64_t> off(std::max<int64_t>(d.ncouplings, 1), 0);
    if (toep) {
        // spectra as stored: whole padded arrays, or their first-axis halves
        std::vector<double> packed;
        for (int64_t k = 0; k < d.ncouplings; ++k) {
            off[k] = (int64_t)packed.size() / 2;
            const int n0 = ts[3 * k], n1 = ts[3 * k + 1], n2 = ts[3 * k + 2];
            if (n0 == 0) continue;
            const int h0 = M.half_spectrum ? n0 / 2 + 1 : n0;
            const double *K = d.coupling + d.coupling_offset[k];
            // a permuted coupling (PermutedTranslation) is expanded here: t[e] = canonical[perm[e]];
            // the per-translation spectra are small next to the moments they multiply
            const int32_t *pm = (d.coupling_rowperm && d.coupling_rowperm[k] >= 0)
                                    ? d.coupling_perm + d.coupling_rowperm[k] : nullptr;
            for (int r = 0; r < n1 * n2; ++r)
                for (int k1 = 0; k1 < h0; ++k1) {
                    const int64_t e = k1 + (int64_t)n0 * r;
                    const int64_t src = pm ? pm[e] : e;
                    packed.push_back(K[2 * src]);
                    packed.push_back(K[2 * src + 1]);
                }
        }
        if (packed.empty()) packed.assign(2, 0.0);
        const int64_t n = (int64_t)packed.size() / 2;
        if (c->precision == H2B_FP64) st = upload_scalars<cdouble>(c, packed.data(), n, &M.cpl);
        else st = upload_scalars<cfloat>(c, packed.data(), n, &M.cpl);
    } else {
        const int fw = cplx ? 2 : 1;
        for (int64_t k = 0; k < d.ncouplings; ++k) off[k] = d.coupling_offset[k] / fw;
        st = upload_far_scalars(c, d.coupling, d.coupling_len / fw, &M.cpl);
        if (st == H2B_OK && c->precision == H2B_FP32 && d.coupling_kind == H2B_COUPLING_DENSE)
            st = build_transposed_couplings(c, d, off);
    }
    if (st) return st;
    int64_t *q;
    CUDA_TRY(c->upload(&q, off.data(), off.size()));
    M.cpl_off = q;
    // permuted dense couplings (PermutedDenseTranslation): the canonical blocks stay shared; per
    // coupling a set [rowperm | rowperm^-1 | colperm | colperm^-1] (n each) that the I2O kernel
    // reads through (identity where a permutation is absent)
    std::vector<int64_t> perm_set;
    if (!toep && d.coupling_rowperm && d.coupling_kind == H2B_COUPLING_DENSE) {
        std::vector<int> sets;
        std::map<std::tuple<int64_t, int64_t, int64_t>, int64_t> made;
        perm_set.assign(std::max<int64_t>(d.ncouplings, 1), -1);
        std::vector<int64_t> nk(std::max<int64_t>(d.ncouplings, 1), -1);  // square: n x n
        for (const h2b_side_desc *sd : {&d.test, &d.trial})
            for (int n = 0; n < sd->nnodes; ++n)
                for (int p = sd->i2o_ptr[n]; p < sd->i2o_ptr[n + 1]; ++p)
                    nk[sd->i2o_coupling[p]] = ncoef_host(*sd, sd->level[n]);
        for (int64_t k = 0; k < d.ncouplings; ++k) {
            const int64_t ro = d.coupling_rowperm[k], co = d.coupling_colperm[k], n = nk[k];
            if ((ro < 0 && co < 0) || n < 0) continue;
            auto it = made.find({ro, co, n});
            if (it != made.end()) {
                perm_set[k] = it->second;
                continue;
            }
            const int64_t base = (int64_t)sets.size();
            sets.resize(base + 4 * n);
            for (int w = 0; w < 2; ++w) {
                const int64_t o = w == 0 ? ro : co;
                int *fw = sets.data() + base + 2 * w * n, *iv = fw + n;
                for (int64_t i = 0; i < n; ++i) fw[i] = o >= 0 ? d.coupling_perm[o + i] : (int)i;
                for (int64_t i = 0; i < n; ++i) iv[fw[i]] = (int)i;
            }
            made[{ro, co, n}] = base;
            perm_set[k] = base;
        }
        if (sets.empty()) sets.assign(1, 0);
        int *pq;
        CUDA_TRY(c->upload(&pq, sets.data(), sets.size()));
        M.perm = pq;
    }
    // per-pair operand offsets for the I2O kernel (both sides; sources live on the other side)
    for (int side = 0; side < 2; ++side) {
        const h2b_side_desc &sd = side == 0 ? d.test : d.trial;
        SideHost &h = side == 0 ? c->test : c->trial;
        const SideHost &o = side == 0 ? c->trial : c->test;
        const int np = sd.i2o_ptr[sd.nnodes];
        std::vector<int64_t> psrc(std::max(np, 1)), pcpl(std::max(np, 1)), pperm(std::max(np, 1), -1);
        for (int p = 0; p < np; ++p) {
            const int src = sd.i2o_src[p];
            psrc[p] = toep ? o.spec_off_host[src] : o.mom_off_host[src];
            pcpl[p] = off[sd.i2o_coupling[p]];
            if (!perm_set.empty()) pperm[p] = perm_set[sd.i2o_coupling[p]];
        }
        CUDA_TRY(c->upload(&q, psrc.data(), psrc.size())); h.d.pair_src = q;
        CUDA_TRY(c->upload(&q, pcpl.data(), pcpl.size())); h.d.pair_cpl = q;
        if (!perm_set.empty()) {
            CUDA_TRY(c->upload(&q, pperm.data(), pperm.size()));
            h.d.pair_perm = q;
        }
        if (toep) {
            st = build_sibling_groups(c, sd, h, o.spec_off_host, off);
            if (st) return st;
        } else if (d.coupling_kind == H2B_COUPLING_DENSE) {
            st = build_group_tiles(c, sd, h, pcpl);
            if (st) return st;
        }
    }
    return build_near(c, d);
}

}  // namespace

// Device address of the no-alloc scratch array on the current device (defined with the array at
// the end of this file); h2b_core_create calls it once so that the array is resident from then on.
h2b_status noalloc_scratch(void **out);

// =============================================================================================
// C ABI
// =============================================================================================
extern "C" {

int32_t h2b_version(void) { return (1 << 16) | 0; }

const char *h2b_last_error(void) { return g_err.c_str(); }

h2b_status h2b_tensor_wait_timeouts(int32_t device, uint32_t *count) {
    if (!count) return fail(H2B_ERR_INVALID, "null argument");
    int ndev = 0;
    CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(H2B_ERR_INVALID, "device %d not present", device);
    DeviceGuard guard(device);
    CUDA_TRY(cudaDeviceSynchronize());
    unsigned v = 0;
    CUDA_TRY(read_umma_timeouts(&v));
    *count = v;
    return H2B_OK;
}

h2b_status h2b_set_tensor_wait_limit(int32_t device, uint32_t limit) {
    int ndev = 0;
    CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(H2B_ERR_INVALID, "device %d not present", device);
    DeviceGuard guard(device);
    CUDA_TRY(cudaDeviceSynchronize());
    CUDA_TRY(set_umma_wait_limit(limit));
    return H2B_OK;
}

h2b_status h2b_core_create(const h2b_map_desc *desc, int32_t device, h2b_core **out) {
    if (!desc || !out) return fail(H2B_ERR_INVALID, "null argument");
    *out = nullptr;
    try {
        h2b_status st = validate(*desc);
        if (st) return st;
        int ndev = 0;
        CUDA_TRY(cudaGetDeviceCount(&ndev));
        if (device < 0 || device >= ndev) return fail(H2B_ERR_INVALID, "device %d not present", device);
        DeviceGuard guard(device);
        (void)cudaGetLastError();  // a non-sticky error left by other code is not this call's
        h2b_core *c = new h2b_core();
        c->device = device;
        c->field = desc->field;
        c->precision = desc->precision;
        c->conj_leaf = desc->conj_leaf_adjoint != 0;
        for (int m = 0; m < 3; ++m) c->alpha[m] = {desc->alpha[m][0], desc->alpha[m][1]};
        st = build_core(c, *desc);
        if (st == H2B_OK) {
            // Load this file's device module on the device now, with the rest of the core's
            // memory: under lazy module loading the no-alloc scratch array is reserved when its
            // module is first loaded, and that must not be the first h2b_farmul_noalloc call.
            void *scratch = nullptr;
            st = noalloc_scratch(&scratch);
        }
        if (st) {
            c->release();
            delete c;
            return st;
        }
        *out = c;
        return H2B_OK;
    } catch (const std::bad_alloc &) {
        return fail(H2B_ERR_NOMEM, "host allocation failed");
    } catch (...) {
        return fail(H2B_ERR_INVALID, "unexpected exception in h2b_core_create");
    }
}

h2b_status h2b_core_destroy(h2b_core *core) {
    if (!core) return H2B_OK;
    DeviceGuard guard(core->device);
    core->release();
    delete core;
    (void)cudaGetLastError();  // teardown reports nothing to later calls
    return H2B_OK;
}

h2b_status h2b_core_get_info(const h2b_core *core, h2b_core_info *out) {
    if (!core || !out) return fail(H2B_ERR_INVALID, "null argument");
    out->device_bytes = core->bytes;
    out->near_entries = core->near_entries;
    out->npairs[0] = core->test.npairs;
    out->npairs[1] = core->trial.npairs;
    out->moment_elems = std::max(core->test.mom_total, core->trial.mom_total);
    out->spectrum_elems = std::max(core->test.spec_total, core->trial.spec_total);
    out->nrows = core->test.ndofs;
    out->ncols = core->trial.ndofs;
    return H2B_OK;
}

h2b_status h2b_workspace_destroy(h2b_workspace *ws) {
    if (!ws) return H2B_OK;
    DeviceGuard guard(ws->core->device);
    if (ws->ev_done) cudaEventSynchronize(ws->ev_done);
    for (void *p : ws->allocs) cudaFree(p);
    if (ws->timeouts) cudaFreeHost(ws->timeouts);
    if (ws->aux) cudaStreamDestroy(ws->aux);
    if (ws->ev_fork) cudaEventDestroy(ws->ev_fork);
    if (ws->ev_join) cudaEventDestroy(ws->ev_join);
    if (ws->ev_far) cudaEventDestroy(ws->ev_far);
    if (ws->ev_done) cudaEventDestroy(ws->ev_done);
    delete ws;
    (void)cudaGetLastError();  // teardown reports nothing to later calls
    return H2B_OK;
}

h2b_status h2b_workspace_create(h2b_core *core, int32_t max_nrhs, h2b_workspace **out) {
    if (!core || !out) return fail(H2B_ERR_INVALID, "null argument");
    if (max_nrhs < 1) return fail(H2B_ERR_INVALID, "max_nrhs must be >= 1");
    *out = nullptr;
    DeviceGuard guard(core->device);
    (void)cudaGetLastError();  // a non-sticky error left by other code is not this call's
    h2b_workspace *ws = new (std::nothrow) h2b_workspace();
    if (!ws) return fail(H2B_ERR_NOMEM, "host allocation failed");
    ws->core = core;
    ws->max_nrhs = max_nrhs;
    const bool cplx = core->field == H2B_COMPLEX;
    const size_t tsz = (cplx ? 2 : 1) * (core->precision == H2B_FP64 ? 8 : 4);
    const size_t ssz = 2 * (core->precision == H2B_FP64 ? 8 : 4);
    const size_t vsz = cplx ? 16 : 8;
    const int64_t mom = std::max(core->test.mom_total, core->trial.mom_total) * max_nrhs;
    const int64_t spec = std::max(core->test.spec_total, core->trial.spec_total) * max_nrhs;
    const int64_t ndof = std::max(core->test.ndofs, core->trial.ndofs) * (int64_t)max_nrhs;
    auto al = [&](void **p, size_t bytes) -> cudaError_t {
        cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
        if (e == cudaSuccess) ws->allocs.push_back(*p);
        return e;
    };
    cudaError_t e = al(&ws->am, mom * tsz);
    if (e == cudaSuccess) e = al(&ws->dm, mom * tsz);
    if (e == cudaSuccess) e = al(&ws->as, spec * ssz);
    if (e == cudaSuccess) e = al(&ws->ds, spec * ssz);
    if (e == cudaSuccess) e = al(&ws->xbuf, ndof * vsz);
    if (e == cudaSuccess) e = al(&ws->ybuf, ndof * vsz);
    if (e == cudaSuccess && !cplx && max_nrhs >= 8)
        e = al(&ws->xnear, (size_t)std::max(core->test.ndofs, core->trial.ndofs) * 16 * sizeof(double));
    if (e == cudaSuccess && cplx && max_nrhs >= 8 && core->dnear.kind == H2B_NEAR_STORED)
        e = al(&ws->xnear, (size_t)std::max(core->test.ndofs, core->trial.ndofs) * near_rhs_block(max_nrhs) * 2 *
                               sizeof(double));
    // the far passes (a chain of dependent launches, the critical path) run on this stream at the
    // device's greatest priority, so their blocks are scheduled ahead of the near field's, which
    // fills the SMs around them
    int prio_least = 0, prio_greatest = 0;
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&ws->aux, cudaStreamNonBlocking, prio_greatest);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ws->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ws->ev_join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ws->ev_far, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ws->ev_done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaHostAlloc((void **)&ws->timeouts, 2 * sizeof(unsigned), cudaHostAllocDefault);
    if (e != cudaSuccess) {
        h2b_workspace_destroy(ws);
        return fail(e == cudaErrorMemoryAllocation ? H2B_ERR_NOMEM : H2B_ERR_CUDA,
                    "workspace allocation failed: %s", cudaGetErrorString(e));
    }
    *out = ws;
    return H2B_OK;
}

}  // extern "C"

namespace {

enum Kind { KIND_MATVEC, KIND_FAR, KIND_NEAR };

struct BusyGuard {
    std::atomic<int> &flag;
    bool ok;
    explicit BusyGuard(std::atomic<int> &f) : flag(f) {
        int expect = 0;
        ok = flag.compare_exchange_strong(expect, 1);
    }
    ~BusyGuard() {
        if (ok) flag.store(0);
    }
};

// I2O of all receiving nodes of side D from the moments / spectra of side A.
h2b_status run_i2o(h2b_core *c, const SideHost &D, const SideHost &A, const FarArgs &fa, cudaStream_t st) {
    const int maxcoef = std::max(A.maxcoef, D.maxcoef);
    const int maxt = std::max(A.maxtsize, D.maxtsize);
    if (D.sib.ngroups > 0) {
        CUDA_TRY(launch_i2o_siblings(c->field == H2B_COMPLEX, c->precision, c->dmap, D.d, D.sib, D.maxslen, fa, st));
        return H2B_OK;
    }
    const bool cplx = c->field == H2B_COMPLEX;
    if (D.grp.nchunks > 0 && i2o_grouped_eligible(cplx, c->precision, c->dmap, c->dmap.ncomp * fa.nrhs, maxcoef)) {
        CUDA_TRY(launch_i2o_grouped(cplx, c->precision, c->dmap, D.d, A.d, D.grp, maxcoef, fa, st));
        return H2B_OK;
    }
    CUDA_TRY(launch_i2o(cplx, c->precision, c->dmap, D.d, A.d, D.d_recv, D.n_recv, fa,
                        maxcoef, maxt, D.maxhalf, st));
    return H2B_OK;
}

// Per-pass device timing (h2b_profile_matvec): after every launch an event is recorded on the
// pass stream and tagged with the pass and its level; the elapsed time between consecutive events
// is that launch's duration on the device.
struct PassTimer {
    std::vector<cudaEvent_t> ev;
    std::vector<std::pair<int, int>> tag;  // (operation, level) of the launch ending at ev[i + 1]
    cudaError_t event(cudaStream_t st) {
        cudaEvent_t e = nullptr;
        cudaError_t r = cudaEventCreate(&e);
        if (r != cudaSuccess) return r;
        ev.push_back(e);
        return cudaEventRecord(e, st);
    }
    cudaError_t start(cudaStream_t st) { return event(st); }
    cudaError_t mark(cudaStream_t st, int op, int level) {
        tag.emplace_back(op, level);
        return event(st);
    }
    ~PassTimer() {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
};

#define PASS_MARK(op, lvl)                                    \
    do {                                                      \
        if (tm) CUDA_TRY(tm->mark(st, (op), (lvl)));          \
    } while (0)

// The far passes (farmul!, src/farinteractions/farmul.jl:47-70) on the arenas of `fa`: leaf
// aggregation, upward transfers, (Toeplitz: forward transforms), I2O, (inverse transforms),
// downward transfers, leaf disaggregation into y. `wait_before_scatter` (optional) orders the final
// scatter after other work on y; `tm` (optional) records each launch's device time.
h2b_status far_passes_fa(h2b_core *c, const FarArgs &fa, const void *x, int64_t ldx, void *y, int64_t ldy,
                         cdouble alpha_eff, cdouble beta, cudaStream_t st, cudaEvent_t wait_before_scatter,
                         PassTimer *tm) {
    const int mode = fa.mode;
    const SideHost &A = mode == H2B_FORWARD ? c->trial : c->test;
    const SideHost &D = mode == H2B_FORWARD ? c->test : c->trial;
    const bool cplx = c->field == H2B_COMPLEX;
    const int pr = c->precision;
    const bool conjc = mode == H2B_ADJOINT && c->conj_leaf;
    const bool toep = c->dmap.coupling_kind == H2B_COUPLING_TOEPLITZ;
    CUDA_TRY(launch_leaf_aggregate(cplx, pr, c->dmap, A.d, A.d_agg_leaves, A.n_agg_leaves, A.maxcoef,
                                   conjc, fa, x, ldx, st));
    PASS_MARK(H2B_PASS_LEAF_AGGREGATE, 0);
    for (const Stage &sg : A.agg_inner) {
        CUDA_TRY(launch_transfer_up(cplx, pr, c->dmap, A.d, sg.d_nodes, sg.n, mode == H2B_ADJOINT, fa,
                                    A.maxcoef, A.maxsep, st));
        PASS_MARK(H2B_PASS_AGGREGATE, sg.level);
    }
    if (toep) {
        CUDA_TRY(launch_toeplitz_in(cplx, pr, c->dmap, A.d, A.d_store, A.n_store, mode == H2B_TRANSPOSE,
                                    fa, A.maxtsize, A.maxaxis, st));
        PASS_MARK(H2B_PASS_MODULATE_IN, 0);
    }
    {
        const h2b_status si = run_i2o(c, D, A, fa, st);
        if (si) return si;
        PASS_MARK(H2B_PASS_I2O, 0);
    }
    if (toep) {
        CUDA_TRY(launch_toeplitz_out(cplx, pr, c->dmap, D.d, D.d_recv, D.n_recv, mode != H2B_TRANSPOSE,
                                     fa, D.maxtsize, D.maxaxis, st));
        PASS_MARK(H2B_PASS_MODULATE_OUT, 0);
    }
    for (const Stage &sg : D.dis_down) {
        CUDA_TRY(launch_transfer_down(cplx, pr, c->dmap, D.d, sg.d_nodes, sg.n, D.d_received, fa,
                                      D.maxcoef, D.maxsep, st));
        PASS_MARK(H2B_PASS_DISAGGREGATE, sg.level);
    }
    if (wait_before_scatter) CUDA_TRY(cudaStreamWaitEvent(st, wait_before_scatter, 0));
    CUDA_TRY(launch_leaf_disaggregate(cplx, pr, c->dmap, D.d, D.d_init_leaves, D.n_init_leaves, conjc,
                                      fa, alpha_eff, beta, y, ldy, st));
    PASS_MARK(H2B_PASS_LEAF_DISAGGREGATE, 0);
    return H2B_OK;
}

h2b_status far_passes(h2b_workspace *ws, int mode, int nrhs, const void *x, int64_t ldx, void *y,
                      int64_t ldy, cdouble alpha_eff, cdouble beta, cudaStream_t st,
                      cudaEvent_t wait_before_scatter, PassTimer *tm = nullptr) {
    const FarArgs fa{mode, nrhs, ws->am, ws->dm, ws->as, ws->ds};
    return far_passes_fa(ws->core, fa, x, ldx, y, ldy, alpha_eff, beta, st, wait_before_scatter, tm);
}

cdouble cmul(cdouble a, cdouble b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }

h2b_status run(h2b_workspace *ws, Kind kind, int32_t mode, int32_t nrhs, const void *x, int64_t ldx,
               void *y, int64_t ldy, const double *alpha, const double *beta, void *stream,
               bool take_busy = true) {
    if (!ws) return fail(H2B_ERR_INVALID, "null workspace");
    if (mode < 0 || mode > 2) return fail(H2B_ERR_INVALID, "mode must be 0, 1 or 2");
    if (nrhs < 1 || nrhs > ws->max_nrhs)
        return fail(H2B_ERR_INVALID, "nrhs = %d outside 1..%d (workspace max_nrhs)", nrhs, ws->max_nrhs);
    if ((alpha == nullptr) != (beta == nullptr))
        return fail(H2B_ERR_INVALID, "alpha and beta must both be given or both be NULL");
    h2b_core *c = ws->core;
    const int64_t nout = mode == H2B_FORWARD ? c->test.ndofs : c->trial.ndofs;
    const int64_t nin = mode == H2B_FORWARD ? c->trial.ndofs : c->test.ndofs;
    if (!x || !y) return fail(H2B_ERR_INVALID, "null x or y");
    if (ldx < nin || ldy < nout) return fail(H2B_ERR_INVALID, "leading dimension smaller than the vector length");
    if (c->field == H2B_REAL && alpha && (alpha[1] != 0.0 || beta[1] != 0.0))
        return fail(H2B_ERR_INVALID, "complex alpha/beta on a real map");
    BusyGuard busy(ws->busy);
    if (take_busy && !busy.ok) return fail(H2B_BUSY, "workspace is in use by another call");
    DeviceGuard guard(c->device);
    (void)cudaGetLastError();  // a non-sticky error left by other code is not this call's
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // serialise with the previous call on this workspace, whatever stream it used; inside a
    // stream capture the captured order does that, and the event of an earlier, uncaptured call
    // cannot be waited on
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CUDA_TRY(cudaStreamIsCapturing(st, &cap));
    if (cap == cudaStreamCaptureStatusNone) CUDA_TRY(cudaStreamWaitEvent(st, ws->ev_done, 0));
    const cdouble a = alpha ? cdouble{alpha[0], alpha[1]} : cdouble{1.0, 0.0};
    const cdouble b = beta ? cdouble{beta[0], beta[1]} : cdouble{0.0, 0.0};
    const cdouble aA = c->alpha[mode];
    const bool cplx = c->field == H2B_COMPLEX;
    const SideHost &rows = c->test;
    const SideHost &cols = c->trial;
    h2b_status s = H2B_OK;
    if (kind == KIND_NEAR) {
        CUDA_TRY(launch_near(cplx, mode, c->dnear, rows.d, cols.d, nrhs, x, ldx, y, ldy, a, b, ws->xnear, st));
    } else if (kind == KIND_FAR) {
        if (!alpha) {
            CUDA_TRY(launch_zero_columns(cplx, nrhs, nout, y, ldy, st));
            s = far_passes(ws, mode, nrhs, x, ldx, y, ldy, aA, cdouble{0.0, 0.0}, st, nullptr);
        } else {
            s = far_passes(ws, mode, nrhs, x, ldx, y, ldy, cmul(aA, a), b, st, nullptr);
        }
    } else {
        // near on the caller's stream, far on the high-priority auxiliary stream; the far leaf
        // scatter waits for the near product, and the caller's stream for the far passes
        CUDA_TRY(cudaEventRecord(ws->ev_fork, st));
        CUDA_TRY(cudaStreamWaitEvent(ws->aux, ws->ev_fork, 0));
        CUDA_TRY(launch_near(cplx, mode, c->dnear, rows.d, cols.d, nrhs, x, ldx, y, ldy, a, b, ws->xnear, st));
        CUDA_TRY(cudaEventRecord(ws->ev_join, st));
        s = far_passes(ws, mode, nrhs, x, ldx, y, ldy, cmul(aA, a), cdouble{1.0, 0.0}, ws->aux, ws->ev_join);
        if (s) return s;
        CUDA_TRY(cudaEventRecord(ws->ev_far, ws->aux));
        CUDA_TRY(cudaStreamWaitEvent(st, ws->ev_far, 0));
    }
    if (s) return s;
    if (cap == cudaStreamCaptureStatusNone) CUDA_TRY(cudaEventRecord(ws->ev_done, st));
    return H2B_OK;
}

}  // namespace

extern "C" {

h2b_status h2b_matvec(h2b_workspace *ws, int32_t mode, int32_t nrhs, const void *x, int64_t ldx,
                      void *y, int64_t ldy, const double *alpha, const double *beta, void *stream) {
    return run(ws, KIND_MATVEC, mode, nrhs, x, ldx, y, ldy, alpha, beta, stream);
}

h2b_status h2b_farmul(h2b_workspace *ws, int32_t mode, int32_t nrhs, const void *x, int64_t ldx,
                      void *y, int64_t ldy, const double *alpha, const double *beta, void *stream) {
    return run(ws, KIND_FAR, mode, nrhs, x, ldx, y, ldy, alpha, beta, stream);
}

h2b_status h2b_nearmul(h2b_workspace *ws, int32_t mode, int32_t nrhs, const void *x, int64_t ldx,
                       void *y, int64_t ldy, const double *alpha, const double *beta, void *stream) {
    return run(ws, KIND_NEAR, mode, nrhs, x, ldx, y, ldy, alpha, beta, stream);
}

// Host arrays in and out: copy x into the workspace's staging buffer, multiply, copy y out, all
// on `stream`; `wait` synchronises the stream before returning (h2b_matvec_host), otherwise the
// workspace's completion event is moved past the copy out so the next call on this workspace
// cannot overwrite the staging buffers early (h2b_matvec_host_async).
static h2b_status matvec_host_impl(h2b_workspace *ws, int32_t mode, int32_t nrhs, const void *x,
                                   int64_t ldx, void *y, int64_t ldy, const double *alpha,
                                   const double *beta, void *stream, bool wait) {
    if (!ws || !x || !y) return fail(H2B_ERR_INVALID, "null argument");
    if (mode < 0 || mode > 2) return fail(H2B_ERR_INVALID, "mode must be 0, 1 or 2");
    if (nrhs < 1 || nrhs > ws->max_nrhs)
        return fail(H2B_ERR_INVALID, "nrhs = %d outside 1..%d (workspace max_nrhs)", nrhs, ws->max_nrhs);
    h2b_core *c = ws->core;
    const int64_t nout = mode == H2B_FORWARD ? c->test.ndofs : c->trial.ndofs;
    const int64_t nin = mode == H2B_FORWARD ? c->trial.ndofs : c->test.ndofs;
    if (ldx < nin || ldy < nout) return fail(H2B_ERR_INVALID, "leading dimension smaller than the vector length");
    const size_t vsz = c->field == H2B_COMPLEX ? 16 : 8;
    BusyGuard busy(ws->busy);
    if (!busy.ok) return fail(H2B_BUSY, "workspace is in use by another call");
    DeviceGuard guard(c->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    CUDA_TRY(cudaStreamWaitEvent(st, ws->ev_done, 0));
    if (wait) CUDA_TRY(copy_umma_timeouts_async(&ws->timeouts[0], st));
    CUDA_TRY(cudaMemcpy2DAsync(ws->xbuf, nin * vsz, x, ldx * vsz, nin * vsz, nrhs, cudaMemcpyHostToDevice, st));
    const bool need_y = beta && (beta[0] != 0.0 || beta[1] != 0.0);
    if (need_y)
        CUDA_TRY(cudaMemcpy2DAsync(ws->ybuf, nout * vsz, y, ldy * vsz, nout * vsz, nrhs, cudaMemcpyHostToDevice, st));
    h2b_status s = run(ws, KIND_MATVEC, mode, nrhs, ws->xbuf, nin, ws->ybuf, nout, alpha, beta, stream,
                       /*take_busy=*/false);
    if (s) return s;
    CUDA_TRY(cudaMemcpy2DAsync(y, ldy * vsz, ws->ybuf, nout * vsz, nout * vsz, nrhs, cudaMemcpyDeviceToHost, st));
    if (wait) {
        CUDA_TRY(copy_umma_timeouts_async(&ws->timeouts[1], st));
        CUDA_TRY(cudaStreamSynchronize(st));
        if (ws->timeouts[1] != ws->timeouts[0])
            return fail(H2B_ERR_CUDA,
                        "a bounded tensor-core wait gave up during this product (%u on the device so far): some "
                        "output tiles were not written; see h2b_tensor_wait_timeouts", ws->timeouts[1]);
    } else {
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        CUDA_TRY(cudaStreamIsCapturing(st, &cap));
        if (cap == cudaStreamCaptureStatusNone) CUDA_TRY(cudaEventRecord(ws->ev_done, st));
    }
    return H2B_OK;
}

h2b_status h2b_matvec_host(h2b_workspace *ws, int32_t mode, int32_t nrhs, const void *x,
                           int64_t ldx, void *y, int64_t ldy, const double *alpha,
                           const double *beta, void *stream) {
    return matvec_host_impl(ws, mode, nrhs, x, ldx, y, ldy, alpha, beta, stream, true);
}

h2b_status h2b_matvec_host_async(h2b_workspace *ws, int32_t mode, int32_t nrhs, const void *x,
                                 int64_t ldx, void *y, int64_t ldy, const double *alpha,
                                 const double *beta, void *stream) {
    return matvec_host_impl(ws, mode, nrhs, x, ldx, y, ldy, alpha, beta, stream, false);
}

h2b_status h2b_profile_matvec(h2b_workspace *ws, int32_t mode, int32_t nrhs, const void *x, int64_t ldx,
                              void *y, int64_t ldy, const double *alpha, const double *beta, void *stream,
                              h2b_pass_time *records, int32_t capacity, int32_t *count) {
    if (!ws || !x || !y || !count || (capacity > 0 && !records)) return fail(H2B_ERR_INVALID, "null argument");
    if (mode < 0 || mode > 2) return fail(H2B_ERR_INVALID, "mode must be 0, 1 or 2");
    if (nrhs < 1 || nrhs > ws->max_nrhs)
        return fail(H2B_ERR_INVALID, "nrhs = %d outside 1..%d (workspace max_nrhs)", nrhs, ws->max_nrhs);
    if ((alpha == nullptr) != (beta == nullptr))
        return fail(H2B_ERR_INVALID, "alpha and beta must both be given or both be NULL");
    h2b_core *c = ws->core;
    const int64_t nout = mode == H2B_FORWARD ? c->test.ndofs : c->trial.ndofs;
    const int64_t nin = mode == H2B_FORWARD ? c->trial.ndofs : c->test.ndofs;
    if (ldx < nin || ldy < nout) return fail(H2B_ERR_INVALID, "leading dimension smaller than the vector length");
    if (c->field == H2B_REAL && alpha && (alpha[1] != 0.0 || beta[1] != 0.0))
        return fail(H2B_ERR_INVALID, "complex alpha/beta on a real map");
    BusyGuard busy(ws->busy);
    if (!busy.ok) return fail(H2B_BUSY, "workspace is in use by another call");
    DeviceGuard guard(c->device);
    (void)cudaGetLastError();  // a non-sticky error left by other code is not this call's
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CUDA_TRY(cudaStreamIsCapturing(st, &cap));
    if (cap != cudaStreamCaptureStatusNone)
        return fail(H2B_ERR_INVALID, "h2b_profile_matvec waits for its events and cannot run inside a stream capture");
    CUDA_TRY(cudaStreamWaitEvent(st, ws->ev_done, 0));
    const cdouble a = alpha ? cdouble{alpha[0], alpha[1]} : cdouble{1.0, 0.0};
    const cdouble b = beta ? cdouble{beta[0], beta[1]} : cdouble{0.0, 0.0};
    PassTimer tm;
    CUDA_TRY(tm.start(st));
    // the passes of h2b_matvec, serialised on the caller's stream so that each has its own interval
    CUDA_TRY(launch_near(c->field == H2B_COMPLEX, mode, c->dnear, c->test.d, c->trial.d, nrhs, x, ldx, y, ldy,
                         a, b, ws->xnear, st));
    CUDA_TRY(tm.mark(st, H2B_PASS_NEAR, 0));
    const h2b_status s = far_passes(ws, mode, nrhs, x, ldx, y, ldy, cmul(c->alpha[mode], a), cdouble{1.0, 0.0},
                                    st, nullptr, &tm);
    if (s) return s;
    CUDA_TRY(cudaEventRecord(ws->ev_done, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    *count = (int32_t)tm.tag.size();
    for (size_t i = 0; i < tm.tag.size() && (int32_t)i < capacity; ++i) {
        float ms = 0.0f;
        CUDA_TRY(cudaEventElapsedTime(&ms, tm.ev[i], tm.ev[i + 1]));
        records[i].pass = tm.tag[i].first;
        records[i].level = tm.tag[i].second;
        records[i].milliseconds = ms;
    }
    return H2B_OK;
}

}  // extern "C"

// =============================================================================================
// Far part in the library's own scratch: h2b_farmul_noalloc.
//
// For callers that cannot allocate device memory when they multiply (their GPU memory belongs to
// another allocator, or allocation is forbidden after start-up): the moment and spectrum arenas
// that a workspace would allocate are carved out of one array compiled into this file instead.
// =============================================================================================
namespace {

// The scratch array (H2B_NOALLOC_SCRATCH_BYTES on every device that loads the library, until the
// process exits). Device code may name it directly; host code must not pass `g_noalloc_scratch`
// itself to a kernel -- on the host that name is only a stand-in, not a device address -- and
// asks the runtime for the address on each device instead (noalloc_scratch below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[H2B_NOALLOC_SCRATCH_BYTES];

}  // namespace

// Device address of the scratch array on the current device. The first lookup on a device loads
// this file's device module there (under lazy module loading), which is when the array's memory is
// reserved; h2b_core_create makes that lookup, so a later call only reads the module's symbol
// table and allocates nothing. The address is not cached across calls: after a device reset the
// module is loaded again at a new address, and a fresh lookup always names the live one.
h2b_status noalloc_scratch(void **out) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
        return fail(e == cudaErrorMemoryAllocation ? H2B_ERR_NOMEM : H2B_ERR_CUDA,
                    "cudaGetSymbolAddress of the no-alloc scratch failed: %s", cudaGetErrorString(e));
    *out = p;
    return H2B_OK;
}

namespace {

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

}  // namespace

extern "C" h2b_status h2b_farmul_noalloc(const h2b_core *core_in, int32_t mode, int32_t nrhs,
                                         const void *x, int64_t ldx, void *y, int64_t ldy,
                                         const double *alpha, const double *beta, void *stream) {
    h2b_core *c = const_cast<h2b_core *>(core_in);
    if (!c) return fail(H2B_ERR_INVALID, "null core");
    if (mode < 0 || mode > 2) return fail(H2B_ERR_INVALID, "mode must be 0, 1 or 2");
    if (nrhs < 1) return fail(H2B_ERR_INVALID, "nrhs must be >= 1");
    if ((alpha == nullptr) != (beta == nullptr))
        return fail(H2B_ERR_INVALID, "alpha and beta must both be given or both be NULL");
    if (!x || !y) return fail(H2B_ERR_INVALID, "null x or y");
    const int64_t nout = mode == H2B_FORWARD ? c->test.ndofs : c->trial.ndofs;
    const int64_t nin = mode == H2B_FORWARD ? c->trial.ndofs : c->test.ndofs;
    if (ldx < nin || ldy < nout) return fail(H2B_ERR_INVALID, "leading dimension smaller than the vector length");
    if (c->field == H2B_REAL && alpha && (alpha[1] != 0.0 || beta[1] != 0.0))
        return fail(H2B_ERR_INVALID, "complex alpha/beta on a real map");
    // scratch layout: aggregation moments, disaggregation moments, then (Toeplitz) both spectra
    const bool cplx = c->field == H2B_COMPLEX;
    const size_t tsz = (cplx ? 2 : 1) * (c->precision == H2B_FP64 ? 8 : 4);
    const size_t ssz = 2 * (c->precision == H2B_FP64 ? 8 : 4);
    const size_t mom = align256((size_t)std::max(c->test.mom_total, c->trial.mom_total) * nrhs * tsz);
    const size_t spec = align256((size_t)std::max(c->test.spec_total, c->trial.spec_total) * nrhs * ssz);
    const size_t need = 2 * mom + 2 * spec;
    if (need > (size_t)H2B_NOALLOC_SCRATCH_BYTES)
        return fail(H2B_ERR_UNSUPPORTED,
                    "h2b_farmul_noalloc: this map needs %zu bytes of scratch for %d right-hand side(s); "
                    "the built-in scratch holds %u bytes (use a workspace and h2b_farmul instead)",
                    need, nrhs, (unsigned)H2B_NOALLOC_SCRATCH_BYTES);
    DeviceGuard guard(c->device);
    (void)cudaGetLastError();  // a non-sticky error left by other code is not this call's
    void *base = nullptr;
    h2b_status s = noalloc_scratch(&base);
    if (s) return s;
    unsigned char *b = static_cast<unsigned char *>(base);
    // Nothing in the scratch needs clearing: every pass overwrites a moment or spectrum slot
    // before any pass reads it (leaf products and first-child / first-pair writes overwrite),
    // so whatever the previous call left there is never read.
    FarArgs fa{mode, nrhs, b, b + mom, b + 2 * mom, b + 2 * mom + spec};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const cdouble aA = c->alpha[mode];
    if (!alpha) {
        CUDA_TRY(launch_zero_columns(cplx, nrhs, nout, y, ldy, st));
        return far_passes_fa(c, fa, x, ldx, y, ldy, aA, cdouble{0.0, 0.0}, st, nullptr, nullptr);
    }
    return far_passes_fa(c, fa, x, ldx, y, ldy, cmul(aA, cdouble{alpha[0], alpha[1]}),
                         cdouble{beta[0], beta[1]}, st, nullptr, nullptr);
}
