// Internal definitions shared by the host orchestration (h2b_api.cu) and the kernels
// (h2b_kernels.cu): scalar types, the device-resident core layout, and kernel launchers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/h2b200.h"

namespace h2b {

// ---------------------------------------------------------------------------------------------
// Scalars. V is the field type of x, y and the near blocks (double or cdouble); T is the far-field
// arithmetic type (double, float, cdouble or cfloat); Toeplitz spectra are complex of T's real type.
// ---------------------------------------------------------------------------------------------
template <class R>
struct Cx {
    R x, y;
};
using cdouble = Cx<double>;
using cfloat = Cx<float>;

// Acc: the arithmetic type of every far-field sum. The FP32 form stores moments, spectra, collections,
// transfers and couplings in FP32 (half the bytes) but accumulates in FP64, so each stored
// intermediate is rounded once instead of once per operation.
template <class T> struct ScalarTraits;
template <> struct ScalarTraits<double> { using Real = double; using Complex = cdouble; using Acc = double; using CAcc = cdouble; static constexpr bool is_complex = false; };
template <> struct ScalarTraits<float> { using Real = float; using Complex = cfloat; using Acc = double; using CAcc = cdouble; static constexpr bool is_complex = false; };
template <> struct ScalarTraits<cdouble> { using Real = double; using Complex = cdouble; using Acc = cdouble; using CAcc = cdouble; static constexpr bool is_complex = true; };
template <> struct ScalarTraits<cfloat> { using Real = float; using Complex = cfloat; using Acc = cdouble; using CAcc = cdouble; static constexpr bool is_complex = true; };

template <class R> __host__ __device__ __forceinline__ Cx<R> operator+(Cx<R> a, Cx<R> b) { return {a.x + b.x, a.y + b.y}; }
template <class R> __host__ __device__ __forceinline__ Cx<R> operator-(Cx<R> a, Cx<R> b) { return {a.x - b.x, a.y - b.y}; }
template <class R> __host__ __device__ __forceinline__ Cx<R> operator*(Cx<R> a, Cx<R> b) {
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <class R> __host__ __device__ __forceinline__ Cx<R> operator*(R a, Cx<R> b) { return {a * b.x, a * b.y}; }
template <class R> __host__ __device__ __forceinline__ Cx<R> &operator+=(Cx<R> &a, Cx<R> b) { a.x += b.x; a.y += b.y; return a; }

__host__ __device__ __forceinline__ double conjg(double a) { return a; }
__host__ __device__ __forceinline__ float conjg(float a) { return a; }
template <class R> __host__ __device__ __forceinline__ Cx<R> conjg(Cx<R> a) { return {a.x, -a.y}; }

template <class T> __host__ __device__ __forceinline__ T sc_zero() { return T{}; }
template <class T> __host__ __device__ __forceinline__ bool is_zero(T a);
template <> __host__ __device__ __forceinline__ bool is_zero(double a) { return a == 0.0; }
template <> __host__ __device__ __forceinline__ bool is_zero(cdouble a) { return a.x == 0.0 && a.y == 0.0; }

// optional conjugation
template <class T> __host__ __device__ __forceinline__ T cj(T a, bool c) { return c ? conjg(a) : a; }

// conversions between the field type V and the far type T (same complexness)
__host__ __device__ __forceinline__ double to_t(double v, double) { return v; }
__host__ __device__ __forceinline__ float to_t(double v, float) { return (float)v; }
__host__ __device__ __forceinline__ cdouble to_t(cdouble v, cdouble) { return v; }
__host__ __device__ __forceinline__ cfloat to_t(cdouble v, cfloat) { return {(float)v.x, (float)v.y}; }
__host__ __device__ __forceinline__ double to_v(double t) { return t; }
__host__ __device__ __forceinline__ double to_v(float t) { return (double)t; }
__host__ __device__ __forceinline__ cdouble to_v(cdouble t) { return t; }
__host__ __device__ __forceinline__ cdouble to_v(cfloat t) { return {(double)t.x, (double)t.y}; }
// widening to the accumulation type and rounding back to the storage type
__host__ __device__ __forceinline__ double wide(double a) { return a; }
__host__ __device__ __forceinline__ double wide(float a) { return (double)a; }
__host__ __device__ __forceinline__ cdouble wide(cdouble a) { return a; }
__host__ __device__ __forceinline__ cdouble wide(cfloat a) { return {(double)a.x, (double)a.y}; }
__host__ __device__ __forceinline__ void narrow(double a, double &o) { o = a; }
__host__ __device__ __forceinline__ void narrow(double a, float &o) { o = (float)a; }
__host__ __device__ __forceinline__ void narrow(cdouble a, cdouble &o) { o = a; }
__host__ __device__ __forceinline__ void narrow(cdouble a, cfloat &o) { o = {(float)a.x, (float)a.y}; }
// moment <-> spectrum
template <class R> __host__ __device__ __forceinline__ Cx<R> to_cx(R a) { return {a, (R)0}; }
template <class R> __host__ __device__ __forceinline__ Cx<R> to_cx(Cx<R> a) { return a; }
template <class R> __host__ __device__ __forceinline__ void from_cx(Cx<R> s, R &out) { out = s.x; }
template <class R> __host__ __device__ __forceinline__ void from_cx(Cx<R> s, Cx<R> &out) { out = s; }
__host__ __device__ __forceinline__ void from_cx(cdouble s, float &out) { out = (float)s.x; }
__host__ __device__ __forceinline__ void from_cx(cdouble s, cfloat &out) { out = {(float)s.x, (float)s.y}; }

// ---------------------------------------------------------------------------------------------
// Device-resident side of a core (all pointers device memory).
// ---------------------------------------------------------------------------------------------
struct DSide {
    int nnodes, nlevels, ndofs;
    int nvalues;             // value_ptr[nnodes]: dof entries held by the leaves
    const int *level, *parent, *sector, *child_ptr, *child, *value_ptr, *value;
    const int *shape;        // [(nlevels+1)*3]
    const int64_t *mom_off;  // [nnodes] moment offset per unit right-hand side (elements of T)
    const int64_t *spec_off; // [nnodes] spectrum offset per unit right-hand side (complex elements)
    const int64_t *coll_off; // [nnodes] leaf collection offsets (elements of T)
    const void *coll;        // T
    const int64_t *tr_off;   // [(nlevels+1)*nsectors] transfer offsets (elements of T)
    const void *tr;          // T
    const int *i2o_ptr, *i2o_src;
    const int64_t *i2o_cpl;   // coupling index of each pair
    const int64_t *pair_src;  // per pair: the source's moment / spectrum offset per unit rhs
    const int64_t *pair_cpl;  // per pair: the coupling's element offset in the coupling array
    const int64_t *pair_perm = nullptr;  // per pair: its permutation set in DMap::perm, -1 none
};

struct DMap {
    int ncomp, dim, nsectors;
    int transfer_kind, coupling_kind;
    int half_spectrum;       // Toeplitz spectra stored as half spectra (real maps, Hermitian couplings)
    int cube_ts;             // > 0: every level's padded Toeplitz arrays are cube_ts^3 (3-D cubes)
    const int64_t *cpl_off;  // [ncouplings] offsets in elements of T (dense/diag) or spectrum (Toeplitz)
    const void *cpl;
    // FP32 dense couplings for the tensor-core I2O: every block transposed, at the same offsets,
    // so that transposed / adjoint products read columns of a stored block like forward ones
    const void *cpl_t = nullptr;
    // every dense block starts on a 16-byte boundary and its columns are whole multiples of 16 bytes:
    // the tensor-core I2O then copies coupling columns with bulk (TMA) copies
    int cpl_vec = 0;
    // permuted dense couplings: sets [rowperm | rowperm^-1 | colperm | colperm^-1], n entries each
    const int *perm = nullptr;
};

// One oriented near operator: for every output leaf (group), the dense blocks that write its rows.
// Blocks are column-major, output rows x input columns, leading dimension near_padded_ld(rows).
struct NearOp {
    int ngroups = 0;
    const int *grp_leaf = nullptr;  // [ngroups] output leaf (every output leaf has a group)
    const int64_t *blk_off = nullptr;  // per block id: element offset in `data`
    // (block, 32-column chunk) work units of each group in block order: {first input value,
    // columns (<= 32), element offset of the chunk's first column in `data` (low, high 32 bits;
    // unused by the matrix-free kernels)}; one independent 16-byte load per unit instead of a
    // chain block -> input leaf -> values
    const int *unit_ptr = nullptr;  // [ngroups+1]
    const int4 *unit = nullptr;
    const void *data = nullptr;     // V
    // (group, 32-row slab) pairs covering every output row: the work items of the complex
    // tensor-core near kernel, one warp each
    int nslabs = 0;
    const int2 *slab = nullptr;
};

struct DNear {
    NearOp fwd;              // N: rows on the test side, columns on the trial side
    NearOp tr;               // N^T (unused when symmetric)
    bool symmetric = false;  // N^T == N: transposed products run on `fwd`
    // matrix-free near field (kind != H2B_NEAR_STORED): entries from the points, no block data
    int kind = 0;
    double wavenumber = 0.0;
    const double *test_pts = nullptr;   // [test ndofs * 3]
    const double *trial_pts = nullptr;  // [trial ndofs * 3]
};

// Sibling groups for the Toeplitz I2O (i2o_sibling_kernel): the receiving children of one parent.
// Record `msg` as the calling thread's error text (h2b_last_error) and return `st`.
h2b_status set_error_text(h2b_status st, const char *msg);

struct SibGroups {
    int ngroups = 0;
    const int *recv = nullptr;         // [ngroups*8] receiving node per child slot, -1 if none
    const int *slen = nullptr;         // [ngroups] stored spectrum length of the group's level
    const int *ptr = nullptr;          // [ngroups+1] into src_off / kof
    const int64_t *src_off = nullptr;  // spectrum offset (per unit rhs) of each source of the union
    const int *kof = nullptr;          // [nentries*8] coupling offset of (source, slot), -1 if no pair
};

// Dense I2O for few right-hand sides, grouped by stored block. The receiving nodes are cut into
// chunks of at most GT_R nodes of one level; a chunk's pairs are listed in tiles, each tile a run of
// pairs that read the same stored (canonical) coupling block, from distinct receiving nodes. One CTA
// per chunk stages a block once per tile and applies it to all of the tile's pairs (the symmetry
// permutations act on the gathered moments and on the output rows), summing into the chunk's
// receiving nodes in shared memory: each pair's block is read once per tile instead of once per pair.
constexpr int GT_R = 16;  // receiving nodes per chunk
constexpr int GT_P = 16;  // pairs per tile
struct GroupTiles {
    int nchunks = 0;
    const int *chunk_ptr = nullptr;      // [nchunks+1] into rcv
    const int *rcv = nullptr;            // receiving nodes, chunk by chunk
    const int *tile_ptr = nullptr;       // [nchunks+1] into tile_pp
    const int *tile_pp = nullptr;        // [ntiles+1] into pair / slot
    const int *pair = nullptr;           // pair index (into the side's pair arrays)
    const unsigned char *slot = nullptr; // receiving node of the pair as its position in the chunk
};

// Per-call arguments of the far passes.
struct FarArgs {
    int mode;     // H2B_FORWARD / H2B_TRANSPOSE / H2B_ADJOINT
    int nrhs;
    void *am;     // aggregation moments (T)
    void *dm;     // disaggregation moments (T)
    void *as;     // aggregation spectra (complex of T's real)
    void *ds;     // disaggregation spectra
};

// ---------------------------------------------------------------------------------------------
// Launchers (h2b_kernels.cu). Each enqueues on `st` and returns the launch error.
// `precision`: 0 = T is FP64, 1 = FP32; `cplx`: field is complex.
// ---------------------------------------------------------------------------------------------
cudaError_t launch_leaf_aggregate(bool cplx, int precision, const DMap &m, const DSide &s,
                                  const int *leaves, int nleaves, int maxcoef, bool conjc,
                                  const FarArgs &fa, const void *x, int64_t ldx, cudaStream_t st);
cudaError_t launch_transfer_up(bool cplx, int precision, const DMap &m, const DSide &s,
                               const int *nodes, int nnodes, bool conjt, const FarArgs &fa,
                               int maxcoef, int maxsep, cudaStream_t st);
cudaError_t launch_toeplitz_in(bool cplx, int precision, const DMap &m, const DSide &s,
                               const int *nodes, int nnodes, bool inverse, const FarArgs &fa,
                               int maxtsize, int maxaxis, cudaStream_t st);
cudaError_t launch_i2o(bool cplx, int precision, const DMap &m, const DSide &recv,
                       const DSide &src, const int *nodes, int nnodes, const FarArgs &fa,
                       int maxcoef, int maxtsize, int maxhalf, cudaStream_t st);
cudaError_t launch_toeplitz_out(bool cplx, int precision, const DMap &m, const DSide &s,
                                const int *nodes, int nnodes, bool inverse, const FarArgs &fa,
                                int maxtsize, int maxaxis, cudaStream_t st);
// Dense I2O of the FP32 form on the tcgen05 tensor cores (h2b_umma.cu): taken when the coupling
// storage is dense and the right-hand sides make at least 4 FP32 columns (MMA N padded to 16).
bool i2o_umma_eligible(bool cplx, int precision, const DMap &m, int nq);
cudaError_t launch_i2o_umma(bool cplx, const DMap &m, const DSide &recv, const DSide &src, const int *nodes,
                            int nnodes, const FarArgs &fa, int maxcoef, cudaStream_t st);
// mbarrier waits of the tensor-core kernels that gave up on the current device (0 in a healthy run)
cudaError_t read_umma_timeouts(unsigned *count);
// the same count copied to host memory in order on `st`
cudaError_t copy_umma_timeouts_async(unsigned *host, cudaStream_t st);
// try_wait attempts of every bounded mbarrier wait on the current device (0: the default)
cudaError_t set_umma_wait_limit(unsigned limit);
cudaError_t launch_i2o_siblings(bool cplx, int precision, const DMap &m, const DSide &recv,
                                const SibGroups &g, int maxslen, const FarArgs &fa, cudaStream_t st);
// The grouped dense I2O (GroupTiles) for W x nq <= GT_MAX_COLS field columns (W = 2 complex);
// wider blocks take the tensor-core I2O (measured on a 65,536-point Laplace map, p = 6, FP32 form:
// grouped 8.5 / 16.8 / 41.5 / 46.6 / 74.6 / 96.2 ms for 1-6 real right-hand sides against
// 98 / 150 / 152 ms for the per-node tile kernel and 84 ms for the tcgen05 kernel from 4 columns
// on; with 5 and 6 columns grouped, the batched-uneven pass did not change).
constexpr int GT_MAX_COLS = 4;
bool i2o_grouped_eligible(bool cplx, int precision, const DMap &m, int nq, int maxcoef);
cudaError_t launch_i2o_grouped(bool cplx, int precision, const DMap &m, const DSide &recv, const DSide &src,
                               const GroupTiles &gt, int maxcoef, const FarArgs &fa, cudaStream_t st);
cudaError_t launch_transfer_down(bool cplx, int precision, const DMap &m, const DSide &s,
                                 const int *nodes, int nnodes, const uint8_t *received,
                                 const FarArgs &fa, int maxcoef, int maxsep, cudaStream_t st);
cudaError_t launch_leaf_disaggregate(bool cplx, int precision, const DMap &m, const DSide &s,
                                     const int *leaves, int nleaves, bool conjc, const FarArgs &fa,
                                     cdouble alpha, cdouble beta, void *y, int64_t ldy,
                                     cudaStream_t st);
cudaError_t launch_near(bool cplx, int mode, const DNear &n, const DSide &test, const DSide &trial,
                        int nrhs, const void *x, int64_t ldx, void *y, int64_t ldy, cdouble alpha,
                        cdouble beta, void *xp, cudaStream_t st);
int64_t near_padded_ld(bool cplx, int n);
// right-hand sides per pass of the complex tensor-core near kernel for a block of `nrhs`
int near_rhs_block(int nrhs);
cudaError_t launch_near_repack(bool cplx, const void *src, const int64_t *src_off, const int *blk_row,
                               const int *blk_col, const DSide &rows, const DSide &cols, void *dst,
                               const int64_t *dst_off, int nblocks, bool transpose, cudaStream_t st);
cudaError_t launch_near_symcheck(bool cplx, const void *src, const int64_t *off, const int *mirror,
                                 const int *blk_row, const DSide &rows, int nblocks, int *flag,
                                 cudaStream_t st);
cudaError_t launch_zero_columns(bool cplx, int nrhs, int64_t n, void *y, int64_t ldy,
                                cudaStream_t st);

}  // namespace h2b
