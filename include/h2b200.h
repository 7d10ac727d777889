/*
 * h2b200.h -- C ABI of the B200 H2 matrix-vector product.
 *
 * The library replaces the execution half of H2Factory.jl's map: the read-only core
 * (`src/maps/core.jl:17-33`), the per-request workspace (`src/maps/workspace.jl:81-113`) and
 * `LinearMaps._unsafe_mul!` on it (`src/maps/abstracth2map.jl:42-86`), i.e. near product + far
 * product (aggregation, I2O, disaggregation) in forward, transpose and adjoint orientation.
 *
 * Everything crossing this boundary is plain C: integer index arrays, scalar arrays, sizes,
 * and opaque handles. Complex scalars are interleaved (re, im) pairs of doubles. Node ids,
 * degree-of-freedom ids and levels follow H2Trees' conventions restated in a flattened form:
 *   - node ids are 0-based, levels are 1-based with the root at level 1;
 *   - a leaf is a node without children;
 *   - `sector` is H2Trees.sector(tree, child), the 0-based slot of a child in its parent.
 * Every entry point returns an h2b_status; on failure `h2b_last_error` gives the text.
 * No C++ exception crosses this boundary.
 */
#ifndef H2B200_H
#define H2B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int h2b_status;
#define H2B_OK 0
#define H2B_ERR_INVALID 1     /* malformed descriptor or argument                              */
#define H2B_ERR_CUDA 2        /* a CUDA runtime call failed                                     */
#define H2B_ERR_NOMEM 3       /* device allocation failed or the memory budget was exceeded     */
#define H2B_BUSY 4            /* the workspace is in use (H2Factory's ConcurrentWorkspaceError) */
#define H2B_ERR_UNSUPPORTED 5 /* valid request the library does not implement                 */

/* Scalar field of x, y, leaf collections, level transfers, couplings and near blocks. */
#define H2B_REAL 0    /* double                        */
#define H2B_COMPLEX 1 /* double complex, (re, im) pairs */

/* Arithmetic of the far field (moments, transfers, couplings). The near field and the final
 * near + far summation always run in the field's FP64 type. */
#define H2B_FP64 0
#define H2B_FP32 1

/* Map orientation, H2Factory's isForward / isTranspose / isAdjoint (src/maps/traits.jl:4-8). */
#define H2B_FORWARD 0
#define H2B_TRANSPOSE 1
#define H2B_ADJOINT 2

/* Level-transfer storage, H2Factory's DenseI2I / SeparableI2I (src/maps/leveltranslator.jl:84-118). */
#define H2B_TRANSFER_DENSE 0
#define H2B_TRANSFER_SEPARABLE 1

/* I2O coupling storage, H2Factory's DenseTranslation / DiagonalTranslation /
 * ToeplitzI2OTranslationTrait (src/farinteractions/i2otranslations/i2otranslationtraits.jl:13-41). */
#define H2B_COUPLING_DENSE 0
#define H2B_COUPLING_DIAGONAL 1
#define H2B_COUPLING_TOEPLITZ 2

/* Near-field storage. H2Factory accepts any matrix-like near operator with the required `mul!`
 * methods (docs/src/near/storage.md:7-14); besides stored dense blocks the library offers point
 * kernels whose entries are computed on the fly from the dof coordinates (no near storage):
 *   LAPLACE    K(x, y) = 1 / (4 pi |x - y|),            0 where x == y;
 *   HELMHOLTZ  K(x, y) = exp(i k |x - y|) / (4 pi |x - y|), 0 where x == y (complex field). */
#define H2B_NEAR_STORED 0
#define H2B_NEAR_LAPLACE 1
#define H2B_NEAR_HELMHOLTZ 2

/*
 * One tree side (test = rows / y, trial = columns / x) with the plans that use it.
 *
 * A side is an aggregation side in one orientation and a disaggregation side in the other:
 * the trial side aggregates for forward maps and disaggregates for transpose/adjoint maps
 * (accessors `aggregationplan`/`disaggregationplan`, src/maps/accessors.jl:232-242).
 */
typedef struct h2b_side_desc {
    /* ---- tree (H2Trees.level/parent/sector/children/values) ---- */
    int32_t nnodes;
    int32_t nlevels;           /* levels are 1..nlevels */
    int32_t root;
    int32_t ndofs;             /* length of x (trial) or y (test)                          */
    const int32_t *level;      /* [nnodes]                                                  */
    const int32_t *parent;     /* [nnodes], -1 at the root                                  */
    const int32_t *sector;     /* [nnodes], 0-based child slot; ignored at the root         */
    const int32_t *child_ptr;  /* [nnodes+1] CSR of children, in H2Trees.children order    */
    const int32_t *child;
    const int32_t *value_ptr;  /* [nnodes+1] CSR of the dofs each leaf owns (empty if inner) */
    const int32_t *value;      /* 0-based dof ids, H2Trees.values order                     */

    /* ---- moment shape per level (index = level, entries 0 unused) ---- */
    const int32_t *shape;      /* [(nlevels+1)*3] moment array extents s1,s2,s3 (1 if unused);
                                  the number of coefficients per component is s1*s2*s3 */

    /* ---- aggregation plan (this side aggregating), levels bottom-up ----
     * H2Trees.aggregationlevels / aggregationnodes / storenode, as consumed by
     * aggregatetree! (src/farinteractions/aggregation.jl:58-92, :241-272). */
    int32_t agg_nstages;
    const int32_t *agg_level;  /* [agg_nstages] level of each stage, deepest first */
    const int32_t *agg_ptr;    /* [agg_nstages+1] */
    const int32_t *agg_node;   /* nodes visited per stage */
    const uint8_t *agg_store;  /* [nnodes] storenode(plan, node): moment read by I2O */

    /* ---- disaggregation plan (this side receiving), levels top-down ----
     * H2Trees.isdisaggregationnode / translatingnodes, as consumed by
     * disaggregatetranslatetree! (src/farinteractions/disaggregation.jl:106-295). */
    int32_t dis_nstages;
    const int32_t *dis_level;  /* [dis_nstages] level of each stage, root side first */
    const int32_t *dis_ptr;    /* [dis_nstages+1] */
    const int32_t *dis_node;
    const uint8_t *dis_isnode; /* [nnodes] isdisaggregationnode(plan, node) */
    const int32_t *i2o_ptr;    /* [nnodes+1] translating partners of each receiving node */
    const int32_t *i2o_src;    /* partner node ids on the OTHER side */
    const int64_t *i2o_coupling; /* coupling index of each pair, already resolved through
                                    couplingkey (src/farinteractions/i2otranslations/i2oprotocol.jl:87-92):
                                    pair (r, t) on the test side uses the block stored for (r, t);
                                    on the trial side it uses the block stored for (t, r). */

    /* ---- leaf collections (test/trialmomentcollections) ----
     * For leaf n: ncomp matrices, each ncoef(level(n)) x nvalues(n), column-major, stored one
     * after the other from element offset coll_offset[n]. -1 for non-leaves. */
    const int64_t *coll_offset;  /* [nnodes] */
    const double *coll;          /* field scalars */
    int64_t coll_len;            /* in field scalars */

    /* ---- level transfers (this side's I2I translator; O2O applies its transpose/adjoint) ----
     * transfers[level(child)][sector(child)] (src/maps/leveltranslator.jl:69-72, :110-116).
     * Dense: one ncoef(level-1) x ncoef(level) column-major matrix.
     * Separable: `dim` per-axis matrices, axis d being shape[level-1][d] x shape[level][d],
     * column-major, axis 1 first (src/maps/leveltranslator.jl:168-265). */
    const int64_t *transfer_offset; /* [(nlevels+1)*nsectors], -1 where absent */
    const double *transfer;
    int64_t transfer_len;        /* in field scalars */
} h2b_side_desc;

/* A complete map (H2Factory's core + the flattened plans that a workspace schedules). */
typedef struct h2b_map_desc {
    int32_t field;          /* H2B_REAL / H2B_COMPLEX */
    int32_t precision;      /* H2B_FP64 / H2B_FP32 far field */
    int32_t ncomp;          /* moment components D of AbstractMoment{D,T} (abstractmoment.jl:6) */
    int32_t dim;            /* rank of each moment component array (1..3) */
    int32_t nsectors;       /* children slots per node, 2^dim for a 2^dim tree */
    int32_t transfer_kind;  /* H2B_TRANSFER_* */
    int32_t coupling_kind;  /* H2B_COUPLING_* */
    int32_t conj_leaf_adjoint; /* leafmul(A, isAdjoint): 1 = ConjugatedCollectionMul,
                                  0 = LinAlgebraMulFunctor (src/maps/functors.jl:206-259) */
    double alpha[3][2];     /* α(A, trait) for forward, transpose, adjoint, as (re, im) */
    h2b_side_desc test;
    h2b_side_desc trial;

    /* ---- I2O couplings (I2OTranslationCollection values, one per stored block) ----
     * Dense: ncoef(level r) x ncoef(level t) column-major block for pair (r, t).
     * Diagonal: ncoef values.
     * Toeplitz: prod(2s-1) complex values of the FFT'd wrap-around kernel (always complex),
     *   in column-major order of the padded array (src/moments/toeplitz/toeplitzmoment.jl:28-30). */
    int64_t ncouplings;
    const int64_t *coupling_offset; /* [ncouplings] in doubles */
    const double *coupling;
    int64_t coupling_len;            /* in doubles */

    /* ---- near field: dense blocks per (test leaf, trial leaf) pair, grouped by test leaf.
     * Block b is nvalues(row) x nvalues(col), column-major, from element offset near_offset[b];
     * rows are H2Trees.values(test, row), columns H2Trees.values(trial, col). This is the
     * BlockSparseMatrix layout of ext/H2BlockSparse/assembly.jl:1-87 for the matrix built by
     * nearinteractions (src/nearinteractions/nearmul.jl:54-111). */
    int32_t near_nrows;               /* number of row groups */
    const int32_t *near_row;          /* [near_nrows] test leaf of each row group */
    const int32_t *near_ptr;          /* [near_nrows+1] */
    const int32_t *near_col;          /* trial leaf of each block */
    const int64_t *near_offset;       /* element offset of each block */
    const double *near;               /* field scalars; host memory unless near_on_device */
    int64_t near_len;                 /* in field scalars */
    int32_t near_on_device;           /* 1: `near` is a device pointer on the core's device */

    /* ---- matrix-free near field (near_kind != H2B_NEAR_STORED): the block structure above
     * (near_nrows, near_row, near_ptr, near_col) still names the near leaf pairs, but `near`,
     * `near_offset` are ignored; entry (i, j) of a block is K(test_points[i], trial_points[j]) for
     * dof ids i, j, with K the kernel of near_kind. Points are host arrays of xyz triples (unused
     * coordinates 0). */
    int32_t near_kind;                /* H2B_NEAR_STORED / H2B_NEAR_LAPLACE / H2B_NEAR_HELMHOLTZ */
    double near_wavenumber;           /* k of the Helmholtz kernel */
    const double *test_points;        /* [test.ndofs * 3] */
    const double *trial_points;       /* [trial.ndofs * 3] */

    /* ---- symmetry-reduced couplings (SymmetryReducedDenseTranslation / PermutedTranslation,
     * src/farinteractions/i2otranslations/symmetryreduceddense.jl:1-60,
     * symmetryreducedcollection.jl:1-40, :150-195): the couplings of one symmetry orbit point at
     * the same canonical data (equal coupling_offset) and read it through 0-based permutations
     * held in coupling_perm:
     *   dense:    t[rowperm[i], colperm[j]] = canonical[i, j];
     *   Toeplitz: t[j] = canonical[rowperm[j]], j the linear index of the padded tensor.
     * coupling_rowperm / coupling_colperm hold each coupling's permutation offset, -1 for the
     * identity; NULL when no coupling is permuted (colperm is unused for Toeplitz). */
    const int64_t *coupling_rowperm;  /* [ncouplings] */
    const int64_t *coupling_colperm;  /* [ncouplings] */
    const int32_t *coupling_perm;
    int64_t coupling_perm_len;
} h2b_map_desc;

typedef struct h2b_core h2b_core;
typedef struct h2b_workspace h2b_workspace;

/* Sizes of a built core, for budgets and reports. */
typedef struct h2b_core_info {
    int64_t device_bytes;   /* device memory held by the core */
    int64_t near_entries;   /* stored near-field scalars */
    int64_t npairs[2];      /* I2O pairs on the test / trial side */
    int64_t moment_elems;   /* moment arena elements per right-hand side */
    int64_t spectrum_elems; /* Toeplitz spectra elements per right-hand side (complex) */
    int32_t nrows;          /* test dofs  */
    int32_t ncols;          /* trial dofs */
} h2b_core_info;

/* Library version, (major << 16) | minor. */
int32_t h2b_version(void);

/* Text of the last failure on the calling thread. */
const char *h2b_last_error(void);

/* Number of waits of the library's tensor-core kernels that gave up on `device` since the library
 * was loaded. Every mbarrier wait inside a kernel is bounded; a wait that runs out adds one here,
 * and its CTA stops, frees its tensor memory and leaves its output tile unwritten. 0 in a healthy
 * run; read it after a product to rule out such a tile. Waits for the device's queued work.
 * No counterpart in the reference: its CPU map has no device-side waits. */
h2b_status h2b_tensor_wait_timeouts(int32_t device, uint32_t *count);

/* Bound of every mbarrier wait of the tensor-core kernels on `device`, in try_wait attempts of at
 * most a microsecond each; 0 restores the default (2^20, about a second). A low bound makes the
 * waits give up, which is how tests exercise
 * the timeout path without faulting or hanging anything: the kernels then stop, wait for the
 * products they issued, free their tensor memory and return, and h2b_matvec_host reports
 * H2B_ERR_CUDA. Waits for the device's queued work. No counterpart in the reference. */
h2b_status h2b_set_tensor_wait_limit(int32_t device, uint32_t limit);

/* Validate `desc`, copy it to `device` and build the read-only core: the CUDA equivalent of
 * building an AbstractH2Core (src/maps/core.jl:17-33). The caller keeps its host arrays. */
h2b_status h2b_core_create(const h2b_map_desc *desc, int32_t device, h2b_core **out);
h2b_status h2b_core_destroy(h2b_core *core);
h2b_status h2b_core_get_info(const h2b_core *core, h2b_core_info *out);

/* ---- map blob: a descriptor as one self-contained, 8-byte aligned byte image, to store a core
 * on disk and load it in another process. The reference keeps its cores inside a Julia session and
 * has no file format; the blob carries the core's read-only data (src/maps/core.jl:1-60) and the
 * plans a workspace is built from (src/maps/workspace.jl:81-100).
 *   h2b_map_blob_write: buf = NULL returns the size in *size; near blocks must be host memory.
 *   h2b_map_blob_read: fills *out with pointers INTO `blob` (keep it alive while *out is used);
 *     checks the layout and every array length, not the contents (h2b_core_create does that).
 *   h2b_core_create_from_blob: read + h2b_core_create. */
h2b_status h2b_map_blob_write(const h2b_map_desc *desc, void *buf, size_t cap, size_t *size);
h2b_status h2b_map_blob_read(const void *blob, size_t bytes, h2b_map_desc *out);
h2b_status h2b_core_create_from_blob(const void *blob, size_t bytes, int32_t device, h2b_core **out);

/* Mutable per-request state (moments, spectra, host staging) for up to `max_nrhs` right-hand
 * sides: H2Workspace(core) / similarworkspace (src/maps/workspace.jl:81-113). Several
 * workspaces may share one core. */
h2b_status h2b_workspace_create(h2b_core *core, int32_t max_nrhs, h2b_workspace **out);
h2b_status h2b_workspace_destroy(h2b_workspace *ws);

/*
 * y = α op(A) x + β y on `nrhs` column-major right-hand sides (device pointers, leading
 * dimensions in scalars), op selected by `mode`; LinearMaps._unsafe_mul! on an H2 map
 * (src/maps/abstracth2map.jl:42-86): near product with (α, β), then far product with (α, 1).
 * `alpha`/`beta` point at (re, im) doubles; both NULL gives the 3-argument mul!(y, A, x).
 * `stream` is a cudaStream_t (NULL = legacy default stream). Asynchronous on `stream`.
 * A second call on a workspace that is still inside a call returns H2B_BUSY.
 */
h2b_status h2b_matvec(h2b_workspace *ws, int32_t mode, int32_t nrhs, const void *x, int64_t ldx,
                      void *y, int64_t ldy, const double *alpha, const double *beta,
                      void *stream);

/* Same product on HOST arrays: copies x in, multiplies, copies y out and synchronizes the
 * stream before returning. This is the call a host-language binding makes for mul!(y, A, x).
 * Returns H2B_ERR_CUDA when a bounded tensor-core wait on the device gave up while the product ran
 * (its output is then incomplete; h2b_tensor_wait_timeouts counts such waits). */
h2b_status h2b_matvec_host(h2b_workspace *ws, int32_t mode, int32_t nrhs, const void *x,
                           int64_t ldx, void *y, int64_t ldy, const double *alpha,
                           const double *beta, void *stream);

/* h2b_matvec_host without the final wait: enqueues on `stream` the copy of x into the workspace,
 * the product and the copy of the result into y, and returns. x and y must stay valid and
 * untouched until the stream has passed this work (synchronize the stream or an event recorded on
 * it); with pinned (page-locked) host memory the copies are asynchronous, so a serving loop that
 * gives each of two workspaces its own stream overlaps one request's copies with another's
 * product. A later call on the same workspace, on any stream, waits for this one's copy out.
 * No counterpart in the reference, whose mul! returns when y is written. */
h2b_status h2b_matvec_host_async(h2b_workspace *ws, int32_t mode, int32_t nrhs, const void *x,
                                 int64_t ldx, void *y, int64_t ldy, const double *alpha,
                                 const double *beta, void *stream);

/* Passes of a product, for h2b_profile_matvec. The far passes follow farmul!
 * (src/farinteractions/farmul.jl:47-70): leaf aggregation, one upward transfer per level, the
 * Toeplitz forward transforms, I2O, the inverse transforms, one downward transfer per level and the
 * leaf disaggregation. */
#define H2B_PASS_NEAR 0
#define H2B_PASS_LEAF_AGGREGATE 1
#define H2B_PASS_AGGREGATE 2        /* upward transfers into the nodes of one level */
#define H2B_PASS_MODULATE_IN 3
#define H2B_PASS_I2O 4
#define H2B_PASS_MODULATE_OUT 5
#define H2B_PASS_DISAGGREGATE 6     /* downward transfers into the nodes of one level */
#define H2B_PASS_LEAF_DISAGGREGATE 7

typedef struct h2b_pass_time {
    int32_t pass;         /* H2B_PASS_* */
    int32_t level;        /* level of the nodes the launch writes; 0 when it spans every level */
    double milliseconds;  /* device time of the launch (CUDA events on the caller's stream) */
} h2b_pass_time;

/* The product of h2b_matvec (same arguments and result) with every pass timed on the device:
 * Diagnostics.profilemul / timedmul! (src/diagnostics/timing.jl:122-160), whose records name an
 * operation, its phase and level. The near pass and the far passes run one after another on
 * `stream` (h2b_matvec overlaps them), an event is recorded after each launch, and the call
 * synchronizes the stream before it returns. Writes up to `capacity` records in launch order and
 * the number of passes in *count. Not allowed inside a stream capture (H2B_ERR_INVALID). */
h2b_status h2b_profile_matvec(h2b_workspace *ws, int32_t mode, int32_t nrhs, const void *x, int64_t ldx,
                              void *y, int64_t ldy, const double *alpha, const double *beta, void *stream,
                              h2b_pass_time *records, int32_t capacity, int32_t *count);

/* Far part only: farmul! (src/farinteractions/farmul.jl:8-70). With alpha = beta = NULL y is
 * zero-filled first (3-argument form); otherwise only leaves that receive a far contribution
 * are updated, y_leaf = α α(A) far + β y_leaf. */
h2b_status h2b_farmul(h2b_workspace *ws, int32_t mode, int32_t nrhs, const void *x, int64_t ldx,
                      void *y, int64_t ldy, const double *alpha, const double *beta,
                      void *stream);

/* Near part only: nearmul! (src/nearinteractions/nearmul.jl:8-14), y = α op(N) x + β y. */
h2b_status h2b_nearmul(h2b_workspace *ws, int32_t mode, int32_t nrhs, const void *x,
                       int64_t ldx, void *y, int64_t ldy, const double *alpha,
                       const double *beta, void *stream);

/* Size of the library's built-in far-field scratch, used by h2b_farmul_noalloc. */
#define H2B_NOALLOC_SCRATCH_BYTES (16u << 20)

/*
 * Far part without a workspace and without any device allocation.
 *
 * This entry point has no counterpart in the reference; it exists for callers that cannot
 * allocate device memory at the time they multiply: a host whose device memory is owned by
 * another allocator (a framework's caching pool that holds the GPU), a real-time loop that
 * forbids allocation after start-up, or a binding that cannot create and keep a workspace.
 * Instead of a workspace's moment and spectrum arenas it uses one scratch array compiled into
 * the library (H2B_NOALLOC_SCRATCH_BYTES per device, held by every GPU that loads the library
 * until the process exits). Same semantics as h2b_farmul on `core`.
 *
 * Limits and rules:
 *   - the map's scratch for `nrhs` right-hand sides (two moment arenas, plus two spectrum arenas
 *     for Toeplitz couplings) must fit in H2B_NOALLOC_SCRATCH_BYTES, else H2B_ERR_UNSUPPORTED;
 *   - the scratch is reserved on a device when the library's device code is loaded there, which
 *     h2b_core_create does (under lazy module loading that load would otherwise happen inside the
 *     first call, and that call would then allocate); each call looks the address up again and
 *     reserves nothing, so the calls also stay valid after a device reset and a new core;
 *   - a failure to reserve the scratch fails h2b_core_create with H2B_ERR_NOMEM;
 *   - all calls on a device share the one array: calls whose work overlaps on the GPU (other
 *     streams, other host threads) race and corrupt each other's results. Serialise them.
 *   - it allocates nothing: no cudaMalloc, no cudaFree, no allocating library routine.
 */
h2b_status h2b_farmul_noalloc(const h2b_core *core, int32_t mode, int32_t nrhs, const void *x,
                              int64_t ldx, void *y, int64_t ldy, const double *alpha,
                              const double *beta, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* H2B200_H */
