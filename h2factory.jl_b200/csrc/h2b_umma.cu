// B1 dense I2O of the FP32 form on the fifth-generation tensor cores (tcgen05, kind::tf32).
//
// Per receiving node r: l_r = sum over its pairs of op(B_pair) m_src (translateintonode!,
// src/farinteractions/traversalhelpers.jl:167-219, with the dense applycouplingkernel! of
// src/farinteractions/i2otranslations/i2otranslationcollection.jl:367-409 and the orientation rule
// of i2oprotocol.jl:87-92). For one receiver this is one GEMM whose K dimension runs over the
// concatenated pairs: D[nc x nq] = [op(B_1) op(B_2) ...] [m_1; m_2; ...].
//
// One CTA per (receiver, 128-row tile of its coefficients, tile of right-hand sides), one CTA per
// SM, warp-specialised; the K dimension streams in chunks of 32 FP32 values through UM_NS stages,
// and every hand-off is an mbarrier (no block barrier inside the loop):
//   * coupling warps (0-3), one thread per tile row: each warp bulk-copies (cp.async.bulk) a
//     quarter of the stored columns that chunk c + 3 reads (column kmap[k] of the pair's block:
//     the column permutation of a symmetry-reduced pair is which column is fetched) into a
//     shared-memory ring; every thread then reads its row of the chunk (rowmap applied by the row
//     it reads), splits the 32 values into TF32 high parts and rounded remainders and writes them
//     into a tensor-memory stage with tcgen05.st. The MMAs take this operand (A) straight from
//     tensor memory. Couplings without whole 16-byte columns are read row by row from global
//     memory into a register ring instead;
//   * moment warps (4-6): cp.async each chunk's source moments into a raw shared-memory ring four
//     chunks ahead, then write them as the B operand, TF32 high parts plus remainders, in the
//     canonical no-swizzle K-major layout (a complex piece is split once for its two rows);
//   * one MMA thread (warp 11): per 8-wide k step the products hi*hi + hi*lo + lo*hi (the lo*lo
//     term is below FP32 rounding), N = 64 columns each, into an FP32 accumulator in tensor memory;
//     one commit per chunk releases both operand stages. A tcgen05.mma costs its issuing thread
//     about 50 cycles whatever its N (measured), so products are made as wide as the block allows;
//   * drain warps (7-10, one per tensor-memory lane quarter): the tensor cores round each
//     accumulation toward zero, so one FP32 accumulator over a whole interaction list loses ~1e-4;
//     accumulators live for 64 values of K (2 chunks) only, two alternate, and each finished one is
//     added into an FP64 sum in tensor memory, which the epilogue rounds once into the FP32 moments.
//
// Complex maps run as real GEMMs: with B = Br + i Bi and m = mr + i mi,
//   [Re l | Im l] = [Br Bi] (interleaved along k) x [[mr, mi]; [-mi, mr]] (interleaved rows),
// so the coupling's interleaved (re, im) storage is the A operand as it lies in memory and each
// moment value feeds two B rows (Re rows (mr, -mi), Im rows (mi, mr)). Adjoint maps conjugate B;
// symmetry-reduced couplings apply their row / column permutations in which rows and columns are
// read. FP32 dense couplings are also stored transposed, so every orientation copies columns.
//
// Every wait on an mbarrier is bounded: a wait that gives up counts itself in a device counter
// (h2b_tensor_wait_timeouts) and sets the CTA's abort flag; every role then leaves its loop, the
// MMA thread waits (with the full bound) for the products it issued, the moment warps for their
// copies, and the CTA frees its tensor memory and returns with its output tile unwritten.

#include "h2b_internal.cuh"

namespace h2b {

namespace {

constexpr int UM_M = 128;         // output rows per tile = tensor-memory lanes
constexpr int UM_KC = 32;         // FP32 K values per chunk: 8 groups of 16 bytes per B row
constexpr int UM_KG = UM_KC / 4;
constexpr int UM_NS = 4;          // operand stages: coupling in tensor memory, moments in shared memory
constexpr int UM_LAG = 4;         // moment copies issued this many chunks ahead of their expansion
constexpr int UM_RS = UM_LAG + 2; // raw moment stages (a slot is rewritten two barriers after its last read)
constexpr uint32_t UM_RAWROW = UM_KC * 4 + 16;  // raw moment row: one chunk's values + 16 bytes of padding
// chunks per accumulation segment: 64 values of K are summed in FP32 (the tensor cores' own
// rounding) before the segment is added to the FP64 sum (measured on the 65,536-point sphere:
// relative error 3.4e-7 at 64 values, 6.5e-7 at 128, 1.2e-6 at 256; time +1 % per halving)
constexpr int UM_SEG = 64 / UM_KC;
// Every hand-off between the roles costs a fixed few hundred cycles whatever the chunk holds
// (measured: with the products removed the kernel ran almost as fast as with them; 32-wide chunks
// ran 27 % faster than 16-wide ones), so chunks are as wide as the tensor-memory and shared-memory
// stages allow.
constexpr int UM_AR = 4;          // coupling column stages in shared memory (bulk-copy path)
constexpr int UM_AI = 4;          // warps that issue a chunk's column copies (KQ / UM_AI columns each)
constexpr int UM_ALA = 3;         // coupling columns copied this many chunks ahead
// 4 coupling, 3 moment, 4 drain, 1 MMA: twelve warps place three on each SM sub-partition, whose
// 16K registers then allow up to 170 per thread (a thirteenth warp would cap them at 128)
constexpr int UM_WARPS = 12;
constexpr int UM_BW = 3;           // moment warps
constexpr int UM_BT = UM_BW * 32;  // moment threads
constexpr int UM_THREADS = UM_WARPS * 32;
constexpr int UM_NT_MAX_REAL = 64;    // right-hand sides per tile, real maps (MMA N = 64)
constexpr int UM_NT_MAX_CPLX = 32;    // complex maps: Re and Im rows make MMA N = 64
constexpr uint32_t UM_LBO = 128;            // bytes between the two 16-byte K halves of a k step
constexpr uint32_t UM_SBO = UM_KG * 128;    // bytes between 8-row groups (4 groups of 128 bytes)
constexpr unsigned UM_SUSPEND_NS = 1000;   // suspend-time hint of one try_wait attempt
constexpr unsigned UM_SPIN = 1u << 20;      // default attempts before a wait gives up (about a second)
constexpr unsigned UM_SPIN_FINAL = 1u << 23;  // the final wait for products already issued

__device__ unsigned int g_umma_timeouts = 0;
__device__ unsigned int g_umma_wait_limit = UM_SPIN;

__device__ __forceinline__ int um_ncoef(const DSide &s, int lvl) {
    return s.shape[3 * lvl] * s.shape[3 * lvl + 1] * s.shape[3 * lvl + 2];
}

__device__ __forceinline__ uint32_t su32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (tcgen05): start address, leading (K) and stride (M/N) byte
// offsets in 16-byte units, version 1 at bits 46-47, no swizzle.
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t addr) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(UM_LBO >> 4) << 16) |
           ((uint64_t)(UM_SBO >> 4) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::tf32: FP32 accumulator (bits 4-5 = 1), A and B TF32 (bits 7-9 and
// 10-12 = 2), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
__device__ __forceinline__ uint32_t tf32_idesc(int mrows, int ncols) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(ncols >> 3) << 17) |
           ((uint32_t)(mrows >> 4) << 24);
}

// byte offset of the 16-byte group (row, kg) in a no-swizzle K-major tile of 16-wide rows
__device__ __forceinline__ uint32_t goff(int row, int kg) {
    return (uint32_t)(row >> 3) * UM_SBO + (uint32_t)kg * UM_LBO + (uint32_t)(row & 7) * 16u;
}

// nearest TF32 value (10 explicit mantissa bits, ties away from zero) as FP32 bits with the 13 low
// mantissa bits cleared: add half of their range to the magnitude, then clear them. Moments and
// couplings are finite and far below the overflow edge.
__device__ __forceinline__ uint32_t tf32_bits(float a) {
    return (__float_as_uint(a) + 0x1000u) & 0xFFFFE000u;
}

// x = hi + lo with hi, lo TF32: the high part and the rounded remainder
__device__ __forceinline__ void split2(float x, uint32_t &hi, uint32_t &lo) {
    hi = tf32_bits(x);
    lo = tf32_bits(x - __uint_as_float(hi));
}

// D (+)= A (tensor memory) * B (shared memory), kind::tf32
__device__ __forceinline__ void umma_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t db, uint32_t idesc,
                                        uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "r"(tmem_a), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(bar)), "r"(bytes) : "memory");
}

// bulk copy global -> this CTA's shared memory, completing `bytes` of the barrier's transaction count
__device__ __forceinline__ void bulk_copy(uint32_t dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(su32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(bar)) : "memory");
}

// bounded wait for the completion of the mbarrier phase with the given parity; false when it gave
// up (counted in g_umma_timeouts). Each attempt suspends the thread until the phase completes or
// UM_SUSPEND_NS pass, so waiting warps leave the issue slots to the warps that work beside them on
// the same SM sub-partition (a spinning wait measured 2-3x slower producers).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, unsigned limit) {
    const uint32_t a = su32(bar);
    for (unsigned it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity), "n"(UM_SUSPEND_NS)
            : "memory");
        if (done) return true;
    }
    atomicAdd(&g_umma_timeouts, 1u);
    return false;
}

// the same wait taken by a whole warp, with one outcome for all its lanes (the warps that go on to
// warp-collective tcgen05.ld / tcgen05.st must not diverge)
__device__ __forceinline__ bool warp_wait(uint64_t *bar, uint32_t parity, unsigned limit) {
    const bool ok = mbar_wait(bar, parity, limit);
    return __all_sync(0xffffffffu, ok);
}

__device__ __forceinline__ bool warp_aborted(volatile int *flag) { return __any_sync(0xffffffffu, *flag != 0); }

// named barrier 1 over the moment warps with an OR vote: every participant gets the same answer
__device__ __forceinline__ bool bar_vote_or(bool v) {
    uint32_t out;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "barrier.cta.red.or.pred q, 1, %2, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(out)
        : "r"((uint32_t)v), "n"(UM_BT)
        : "memory");
    return out != 0;
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
        "%13, %14, %15, %16};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
        "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7])
                 : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// element copy global -> shared; ok = false writes zeros (src is then not read)
template <int EB>
__device__ __forceinline__ void cp_elem(uint32_t dst, const void *src, bool ok) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(dst), "l"(src), "n"(EB), "r"(ok ? EB : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_commit_group() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_wait_group() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// One chunk of a tile row (UM_KC FP32 values; complex: (re, im) of op(B)[row, k] along k' = 2k,
// 2k + 1, conjugated for adjoint maps) split into TF32 high parts and remainders and written to the
// row's tensor-memory lane: hi at columns [ta, ta + UM_KC), lo after them. Values past the block
// (element index >= kv) are zero.
template <int W>
__device__ __forceinline__ void store_split(uint32_t ta, const float (&v)[UM_KC], int kv, bool adj) {
#pragma unroll
    for (int h = 0; h < UM_KC / 16; ++h) {
        uint32_t hi[16], lo[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            const int j = 16 * h + e;
            float x = (j / W) < kv ? v[j] : 0.0f;
            if (W == 2 && adj && (j & 1)) x = -x;
            split2(x, hi[e], lo[e]);
        }
        tmem_st16(ta + 16u * h, hi);
        tmem_st16(ta + UM_KC + 16u * h, lo);
    }
    tmem_wait_st();
}

template <class T> struct UmScalar;
template <> struct UmScalar<float> {
    static constexpr int W = 1;  // FP32 values per element
};
template <> struct UmScalar<cfloat> {
    static constexpr int W = 2;
};

// The operands of one pair with the permutations of a symmetry-reduced coupling (sets
// [rowperm | rowperm^-1 | colperm | colperm^-1]) resolved.
template <class T>
struct UmPair {
    const T *B;         // coupling block
    const T *X;         // source moments of the tile's first right-hand side, column-major snc x nq
    int snc;            // source coefficients
    int nk;             // K chunks
    const int *rowmap;  // output row -> row of the (forward or transposed) stored block, or null
    const int *kmap;    // k -> column of the (forward or transposed) stored block, or null
    bool vec;           // the moment columns start on 16-byte boundaries: whole 16-byte copies
};

template <class T>
__device__ __forceinline__ UmPair<T> um_pair(const DMap &m, const DSide &r, const DSide &t, int p, int nc,
                                             bool fwd, int nrhs, int q0, const T *am) {
    constexpr int W = UmScalar<T>::W;
    UmPair<T> u;
    u.snc = um_ncoef(t, t.level[r.i2o_src[p]]);
    u.nk = (W * u.snc + UM_KC - 1) / UM_KC;
    // transposed and adjoint products read the transposed copy: column kmap[k] of the stored block
    u.B = static_cast<const T *>(fwd ? m.cpl : m.cpl_t) + r.pair_cpl[p];
    u.X = am + r.pair_src[p] * nrhs + (int64_t)q0 * u.snc;
    const int64_t ps = r.pair_perm ? r.pair_perm[p] : -1;
    u.rowmap = nullptr;
    u.kmap = nullptr;
    // both permutations act on the stored block, so the moments are read in their own order:
    if (ps >= 0) {
        if (fwd) {  // t[rp[i], cp[j]] = M[i, j]: out[i] += sum_j M[rp^-1[i], cp^-1[j]] x[j]
            u.rowmap = m.perm + ps + nc;
            u.kmap = m.perm + ps + 3 * u.snc;
        } else {    // out[j] += sum_i op(M)[cp^-1[j], rp^-1[i]] x[i]
            u.rowmap = m.perm + ps + 3 * u.snc;
            u.kmap = m.perm + ps + u.snc;
        }
    }
    constexpr int V = 16 / (int)sizeof(T);  // elements per 16 bytes
    u.vec = (r.pair_src[p] * nrhs + (int64_t)q0 * u.snc) % V == 0 && u.snc % V == 0;
    return u;
}

__device__ __forceinline__ float2 ldg2(const cfloat *p) { return __ldg(reinterpret_cast<const float2 *>(p)); }

}  // namespace

template <class T>
__global__ void __maxnreg__(168)
i2o_umma_kernel(DMap m, DSide r, DSide t, const int *__restrict__ nodes, int mode, int nrhs, int qt_max,
                const T *__restrict__ am, T *__restrict__ dm) {
    constexpr int W = UmScalar<T>::W;
    constexpr int EB = sizeof(T);        // bytes per element (4 real, 8 complex)
    constexpr int KQ = UM_KC / W;        // elements along k per chunk
    extern __shared__ __align__(128) unsigned char um_smem[];
    __shared__ uint64_t a_full[UM_NS], b_full[UM_NS], empty[UM_NS], ar_full[UM_AI][UM_AR], ar_empty[UM_AR];
    __shared__ uint64_t acc_full[2], acc_empty[2], fin;
    __shared__ uint32_t tmem_slot;
    __shared__ int nchunks_s;
    __shared__ volatile int abort_s;

    const int node = nodes[blockIdx.x];
    const int nc = um_ncoef(r, r.level[node]);
    const int m0 = blockIdx.y * UM_M;
    const int nq = m.ncomp * nrhs;
    const int q0 = blockIdx.z * qt_max;
    if (m0 >= nc || q0 >= nq) return;  // whole CTA, before any barrier
    const int mt = min(UM_M, nc - m0);
    const int qt = min(qt_max, nq - q0);
    const int np = ((W * qt_max + 15) / 16) * 16;   // MMA N: B rows (real: q; complex: Re rows, then Im rows)
    const int p0 = r.i2o_ptr[node], p1 = r.i2o_ptr[node + 1];
    T *out = dm + r.mom_off[node] * nrhs;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (p0 == p1) {
        for (int o = tid; o < mt * qt; o += UM_THREADS) out[(int64_t)(q0 + o / mt) * nc + m0 + o % mt] = T{};
        return;
    }
    const bool fwd = mode == H2B_FORWARD, adj = mode == H2B_ADJOINT;
    const unsigned limit = g_umma_wait_limit;

    // tensor memory: two FP32 accumulators of np columns (segments alternate between them), the
    // FP64 sum (two columns per value), then UM_NS coupling stages of 2 UM_KC columns (hi, lo)
    const uint32_t col_master = 2 * (uint32_t)np;
    const uint32_t col_a = 4 * (uint32_t)np;
    const uint32_t need = col_a + UM_NS * 2 * UM_KC;
    const uint32_t ncols = need <= 64 ? 64u : (need <= 128 ? 128u : (need <= 256 ? 256u : 512u));
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_slot)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < UM_NS; ++s) {
            mbar_init(&a_full[s], 128);
            mbar_init(&b_full[s], UM_BT);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&acc_full[a], 1);
            mbar_init(&acc_empty[a], 128);
        }
        for (int a = 0; a < UM_AR; ++a) {
            for (int w = 0; w < UM_AI; ++w) mbar_init(&ar_full[w][a], 1);
            mbar_init(&ar_empty[a], 128);
        }
        mbar_init(&fin, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        nchunks_s = 0;
        abort_s = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    {  // chunks of the whole interaction list
        int mine = 0;
        for (int p = p0 + tid; p < p1; p += UM_THREADS) mine += (W * um_ncoef(t, t.level[r.i2o_src[p]]) + UM_KC - 1) / UM_KC;
        if (mine) atomicAdd(&nchunks_s, mine);
        __syncthreads();
    }
    const int C = nchunks_s;
    const int G = (C + UM_SEG - 1) / UM_SEG;
    const uint32_t smem0 = su32(um_smem);
    const uint32_t b_stage_bytes = 2u * (uint32_t)np * (UM_KC * 4);  // hi then lo, canonical layout
    const uint32_t raw0 = smem0 + UM_NS * b_stage_bytes;
    const uint32_t raw_stage_bytes = (uint32_t)qt_max * UM_RAWROW;
    const uint32_t acol_bytes = (uint32_t)nc * EB;                 // one stored coupling column
    const uint32_t astage_bytes = ((uint32_t)KQ * acol_bytes + 127u) & ~127u;
    const uint32_t araw0 = raw0 + ((UM_RS * raw_stage_bytes + 127u) & ~127u);

    if (warp < 4 && m.cpl_vec) {
        // ---------------- coupling warps, bulk-copy path ----------------
        // Per chunk, lane j of issuing warp w copies column kmap[k0 + w KQ / UM_AI + j] of the pair's
        // stored block (nc contiguous values) into a shared-memory stage with a bulk copy, UM_ALA
        // chunks ahead (each issuing warp completes its own barrier of the stage); every
        // thread then reads its own row of those columns, so the scattered accesses of a permuted
        // block stay in shared memory and global memory is read in whole columns.
        const int row = 32 * warp + lane;   // tile row = tensor-memory lane
        const bool live = row < mt;
        const uint32_t tl = tmem + ((uint32_t)(32 * warp) << 16);
        int lp = p0, lk = 0;  // consumption cursor
        UmPair<T> lu = um_pair<T>(m, r, t, p0, nc, fwd, nrhs, q0, am);
        int brow = live ? (lu.rowmap ? lu.rowmap[m0 + row] : m0 + row) : 0;
        int ip = p0, ik = 0, ic = 0;  // copy cursor (issuing warps)
        UmPair<T> iu = lu;
        constexpr int JW = KQ / UM_AI;  // columns copied by each issuing warp
        const int jw = warp * JW;       // this warp's first column of a chunk
        const bool issuer = warp < UM_AI;
        int kcol = 0;  // lane j: stored column of the copy chunk's k = ik KQ + jw + j
        auto fetch_col = [&]() {
            const int k = min(ik * KQ + jw + lane, iu.snc - 1);
            kcol = iu.kmap ? __ldg(iu.kmap + k) : k;
        };
        auto issue = [&]() -> bool {  // issuing warp: its columns of chunk ic
            const int st = ic % UM_AR;
            if (ic >= UM_AR && !warp_wait(&ar_empty[st], ((ic / UM_AR) - 1) & 1, limit)) return false;
            const int nv = max(0, min(JW, iu.snc - ik * KQ - jw));
            const uint32_t dst = araw0 + (uint32_t)st * astage_bytes + (uint32_t)jw * acol_bytes;
            if (lane == 0) mbar_expect_tx(&ar_full[warp][st], (uint32_t)nv * acol_bytes);
            __syncwarp();
            if (lane < nv)
                bulk_copy(dst + (uint32_t)lane * acol_bytes, iu.B + (int64_t)kcol * nc, acol_bytes, &ar_full[warp][st]);
            __syncwarp();
            ++ic;
            if (++ik == iu.nk) {
                ik = 0;
                if (++ip < p1) iu = um_pair<T>(m, r, t, ip, nc, fwd, nrhs, q0, am);
            }
            if (ip < p1) fetch_col();
            return true;
        };
        int cw = 0;  // chunks whose columns this warp has waited for
        if (issuer) {
            fetch_col();
            for (int u = 0; u < UM_ALA && ic < C; ++u)
                if (!issue()) abort_s = 1;
        }
        for (int c = 0; c < C; ++c) {
            if (warp_aborted(&abort_s)) break;
            if (issuer && ic < C && !issue()) {
                abort_s = 1;
                break;
            }
            const int st = c % UM_AR;
            bool landed = true;
#pragma unroll
            for (int w = 0; w < UM_AI; ++w) landed = landed && warp_wait(&ar_full[w][st], (c / UM_AR) & 1, limit);
            if (!landed) {
                abort_s = 1;
                break;
            }
            const int kv = live ? min(KQ, lu.snc - lk * KQ) : 0;
            const uint32_t src = araw0 + (uint32_t)st * astage_bytes + (uint32_t)brow * EB;
            float v[UM_KC];
#pragma unroll
            for (int j = 0; j < KQ; ++j) {
                if constexpr (W == 2) {
                    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];"
                                 : "=f"(v[2 * j]), "=f"(v[2 * j + 1])
                                 : "r"(src + (uint32_t)j * acol_bytes));
                } else {
                    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v[j]) : "r"(src + (uint32_t)j * acol_bytes));
                }
            }
            mbar_arrive(&ar_empty[st]);
            if (++lk == lu.nk) {
                lk = 0;
                if (++lp < p1) {
                    lu = um_pair<T>(m, r, t, lp, nc, fwd, nrhs, q0, am);
                    brow = live ? (lu.rowmap ? lu.rowmap[m0 + row] : m0 + row) : 0;
                }
            }
            const int s = c % UM_NS;
            if (c >= UM_NS && !warp_wait(&empty[s], ((c / UM_NS) - 1) & 1, limit)) {
                abort_s = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t ta = tl + col_a + (uint32_t)s * (2u * UM_KC);
            store_split<W>(ta, v, kv, adj);
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            mbar_arrive(&a_full[s]);
            cw = c + 1;
        }
        if (issuer) {
            // bulk copies issued but not consumed (after a wait gave up) still write this CTA's
            // shared memory: wait for this warp's, with the full bound, before the CTA can exit
            for (int cc = cw; cc < ic; ++cc) mbar_wait(&ar_full[warp][cc % UM_AR], (cc / UM_AR) & 1, UM_SPIN_FINAL);
        }
    } else if (warp < 4) {
        // ---------------- coupling warps: A operand into tensor memory ----------------
        const int row = 32 * warp + lane;   // tile row = tensor-memory lane
        const bool live = row < mt;
        const uint32_t tl = tmem + ((uint32_t)(32 * warp) << 16);
        // load cursor: pair lp, chunk lk, the pair's operands and this thread's row of op(B), one
        // chunk ahead; every load reads a valid address (clamped row and k) and the values past the
        // block are zeroed when the chunk is split, so no instruction waits on a load early
        int lp = p0, lk = 0;
        UmPair<T> lu = um_pair<T>(m, r, t, p0, nc, fwd, nrhs, q0, am);
        int brow = live ? (lu.rowmap ? lu.rowmap[m0 + row] : m0 + row) : 0;
        float ra[2][UM_KC];
        int kv[2];    // valid elements of each buffered chunk (0 for rows past the tile)
        int km[KQ];   // stored-block indices of the next chunk's k (its permutation, fetched a chunk ahead)
        auto fetch_map = [&]() {
#pragma unroll
            for (int j = 0; j < KQ; ++j) {
                const int k = min(lk * KQ + j, lu.snc - 1);
                km[j] = lu.kmap ? __ldg(lu.kmap + k) : k;
            }
        };
        auto load = [&](float (&v)[UM_KC], int &nvalid) {
            const int k0 = lk * KQ;
            nvalid = live ? min(KQ, lu.snc - k0) : 0;
#pragma unroll
            for (int j = 0; j < KQ; ++j) {
                const int k = km[j];
                const T *src = lu.B + brow + (int64_t)k * nc;
                if constexpr (W == 2) {
                    const float2 x = ldg2(src);
                    v[2 * j] = x.x;
                    v[2 * j + 1] = x.y;
                } else {
                    v[j] = __ldg(src);
                }
            }
            if (++lk == lu.nk) {
                lk = 0;
                if (++lp < p1) {
                    lu = um_pair<T>(m, r, t, lp, nc, fwd, nrhs, q0, am);
                    brow = live ? (lu.rowmap ? lu.rowmap[m0 + row] : m0 + row) : 0;
                }
            }
            if (lp < p1) fetch_map();
        };
        fetch_map();
        load(ra[0], kv[0]);
        for (int c0 = 0; c0 < C; c0 += 2) {
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int c = c0 + u;
                if (c >= C || warp_aborted(&abort_s)) break;
                if (c + 1 < C) load(ra[u ^ 1], kv[u ^ 1]);
                const int s = c % UM_NS;
                if (c >= UM_NS && !warp_wait(&empty[s], ((c / UM_NS) - 1) & 1, limit)) {
                    abort_s = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t ta = tl + col_a + (uint32_t)s * (2u * UM_KC);
                store_split<W>(ta, ra[u], kv[u], adj);
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                mbar_arrive(&a_full[s]);
            }
            if (warp_aborted(&abort_s)) break;
        }
    } else if (warp < 4 + UM_BW) {
        // ---------------- moment warps: B operand into shared memory ----------------
        const int bt = tid - 128;
        // copy cursor (pair cp_, chunk ck); a chunk's raw moments are qt_max rows of 64 bytes, copied
        // as 16-byte pieces (consecutive threads: consecutive pieces of a row), element by element
        // where a column is not 16-byte aligned or the chunk runs past the pair's coefficients
        int cp_ = p0, ck = 0;
        UmPair<T> cu = um_pair<T>(m, r, t, p0, nc, fwd, nrhs, q0, am);
        constexpr int EV = 16 / EB;  // elements per piece
        auto issue = [&](int ci) {
            const uint32_t rb = raw0 + (uint32_t)(ci % UM_RS) * raw_stage_bytes;
            const int k0 = ck * KQ;
            for (int pc = bt; pc < qt_max * UM_KG; pc += UM_BT) {
                const int q = pc / UM_KG, kg = pc % UM_KG, kp = k0 + kg * EV;
                const uint32_t dst = rb + (uint32_t)q * UM_RAWROW + (uint32_t)kg * 16;
                const T *src = cu.X + (int64_t)q * cu.snc + kp;
                if (cu.vec && q < qt && kp + EV <= cu.snc) {
                    cp_elem<16>(dst, src, true);
                } else {
#pragma unroll
                    for (int e = 0; e < EV; ++e) {
                        const bool ok = q < qt && kp + e < cu.snc;
                        cp_elem<EB>(dst + (uint32_t)(e * EB), ok ? src + e : cu.X, ok);
                    }
                }
            }
            if (++ck == cu.nk) {
                ck = 0;
                if (++cp_ < p1) cu = um_pair<T>(m, r, t, cp_, nc, fwd, nrhs, q0, am);
            }
        };
        for (int c = 0; c < UM_LAG && c < C; ++c) {
            issue(c);
            cp_commit_group();
        }
        // rows past the right-hand sides' rows (real tiles whose width is not a multiple of 16)
        // are zero in every stage, written once
        for (int o = bt; o < UM_NS * 2 * (np - W * qt_max) * UM_KG; o += UM_BT) {
            const int rr = W * qt_max + (o / UM_KG) % (np - W * qt_max), kg = o % UM_KG;
            const int sh = o / (UM_KG * (np - W * qt_max));  // stage and hi/lo half
            asm volatile("st.shared.v4.b32 [%0], {%1, %1, %1, %1};" ::"r"(smem0 + (uint32_t)sh * ((uint32_t)np * UM_KC * 4) +
                                                                         goff(rr, kg)),
                         "r"(0u));
        }
        const int npieces = qt_max * UM_KG;  // 16-byte pieces of the raw tile
        const int q0p = bt % qt_max, kg0 = bt / qt_max;
        for (int c = 0; c < C; ++c) {
            const int ci = c + UM_LAG;
            if (ci < C) issue(ci);
            cp_commit_group();
            cp_wait_group<UM_LAG>();  // this thread's copies of chunk c have landed
            // ... and everyone's; the vote makes the stop decision the same for all moment threads
            // (a thread that left the loop alone would leave the others waiting at this barrier)
            if (bar_vote_or(abort_s != 0)) break;
            const int s = c % UM_NS;
            // the expanded stage was last read by the products of chunk c - UM_NS
            if (c >= UM_NS && !mbar_wait(&empty[s], ((c / UM_NS) - 1) & 1, limit)) {
                abort_s = 1;  // the stage may still be read: leave it; the next vote stops the loop
                continue;
            }
            const uint32_t rb = raw0 + (uint32_t)(c % UM_RS) * raw_stage_bytes;
            const uint32_t hb = smem0 + (uint32_t)s * b_stage_bytes;
            const uint32_t lb = hb + (uint32_t)np * (UM_KC * 4);
            // raw pieces bt, bt + UM_BT, ... as (row q, k group kg), rows fastest: a quarter-warp
            // reads 8 rows of one k group and writes 8 consecutive rows of the expanded tile
            // (conflict-free); a complex piece (mr, mi) of two k is split once and written to
            // both its rows, Re (mr, -mi) and Im (mi, mr): negation is exact in TF32 parts
            int q = q0p, kg = kg0;
            for (int pc = bt; pc < npieces; pc += UM_BT) {
                if (pc != bt) {
                    q += UM_BT;
                    while (q >= qt_max) {
                        q -= qt_max;
                        ++kg;
                    }
                }
                float w[4];
                asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                             : "=f"(w[0]), "=f"(w[1]), "=f"(w[2]), "=f"(w[3])
                             : "r"(rb + (uint32_t)q * UM_RAWROW + (uint32_t)kg * 16));
                uint32_t h[4], l[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) split2(w[e], h[e], l[e]);
                const uint32_t o = goff(q, kg);
                if constexpr (W == 1) {
                    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(hb + o), "r"(h[0]), "r"(h[1]),
                                 "r"(h[2]), "r"(h[3]));
                    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(lb + o), "r"(l[0]), "r"(l[1]),
                                 "r"(l[2]), "r"(l[3]));
                } else {
                    constexpr uint32_t S = 0x80000000u;
                    const uint32_t oi = goff(qt_max + q, kg);
                    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(hb + o), "r"(h[0]), "r"(h[1] ^ S),
                                 "r"(h[2]), "r"(h[3] ^ S));
                    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(lb + o), "r"(l[0]), "r"(l[1] ^ S),
                                 "r"(l[2]), "r"(l[3] ^ S));
                    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(hb + oi), "r"(h[1]), "r"(h[0]),
                                 "r"(h[3]), "r"(h[2]));
                    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(lb + oi), "r"(l[1]), "r"(l[0]),
                                 "r"(l[3]), "r"(l[2]));
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive(&b_full[s]);
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    } else if (warp < UM_WARPS - 1) {
        // ---------------- drain warps: FP64 sum of the segments, then the epilogue ----------------
        const int lq = warp & 3;
        const int row = 32 * lq + lane;
        const uint32_t tl = tmem + ((uint32_t)(32 * lq) << 16);
        bool ok = true;
        for (int g = 0; g < G; ++g) {
            const int a = g & 1;
            if (!warp_wait(&acc_full[a], (g >> 1) & 1, limit)) {
                abort_s = 1;
                ok = false;
                break;
            }
            if (warp_aborted(&abort_s)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (int j = 0; j < np; j += 16) {
                uint32_t f[16], w0[16], w1[16];
                tmem_ld16(tl + (uint32_t)(a * np + j), f);
                if (g > 0) {
                    tmem_ld16(tl + col_master + 2u * (uint32_t)j, w0);
                    tmem_ld16(tl + col_master + 2u * (uint32_t)j + 16u, w1);
                }
                tmem_wait_ld();
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    uint32_t &lo = e < 8 ? w0[2 * e] : w1[2 * (e - 8)];
                    uint32_t &hi = e < 8 ? w0[2 * e + 1] : w1[2 * (e - 8) + 1];
                    const double prev = g > 0 ? __hiloint2double((int)hi, (int)lo) : 0.0;
                    const double v = prev + (double)__uint_as_float(f[e]);
                    lo = (uint32_t)__double2loint(v);
                    hi = (uint32_t)__double2hiint(v);
                }
                tmem_st16(tl + col_master + 2u * (uint32_t)j, w0);
                tmem_st16(tl + col_master + 2u * (uint32_t)j + 16u, w1);
            }
            tmem_wait_st();
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            mbar_arrive(&acc_empty[a]);
        }
        if (ok && !warp_aborted(&abort_s)) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (int j8 = 0; j8 * 8 < qt; ++j8) {
                uint32_t wr[16], wi[16];
                tmem_ld16(tl + col_master + 2 * (uint32_t)(8 * j8), wr);
                if constexpr (W == 2) tmem_ld16(tl + col_master + 2 * (uint32_t)(qt_max + 8 * j8), wi);
                tmem_wait_ld();
                if (row < mt) {
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        const int q = 8 * j8 + e;
                        if (q >= qt) break;
                        const double re = __hiloint2double((int)wr[2 * e + 1], (int)wr[2 * e]);
                        T *o = out + (int64_t)(q0 + q) * nc + m0 + row;
                        if constexpr (W == 2) {
                            const double im = __hiloint2double((int)wi[2 * e + 1], (int)wi[2 * e]);
                            *o = T{(float)re, (float)im};
                        } else {
                            *o = (float)re;
                        }
                    }
                }
            }
        }
    } else if (lane == 0) {
        // ---------------- MMA thread: six products of N = np columns per chunk ----------------
        const uint32_t idesc = tf32_idesc(UM_M, np);
        for (int c = 0; c < C; ++c) {
            const int s = c % UM_NS, g = c / UM_SEG, a = g & 1;
            if (c % UM_SEG == 0 && g >= 2 && !mbar_wait(&acc_empty[a], ((g >> 1) - 1) & 1, limit)) abort_s = 1;
            if (!abort_s && !mbar_wait(&a_full[s], (c / UM_NS) & 1, limit)) abort_s = 1;
            if (!abort_s && !mbar_wait(&b_full[s], (c / UM_NS) & 1, limit)) abort_s = 1;
            if (abort_s) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t d = tmem + (uint32_t)(a * np);
            const uint32_t ta = tmem + col_a + (uint32_t)s * (2u * UM_KC);
            const uint32_t bh = smem0 + (uint32_t)s * b_stage_bytes, bl = bh + (uint32_t)np * (UM_KC * 4);
#pragma unroll
            for (int j = 0; j < UM_KC / 8; ++j) {
                const uint64_t dbh = kmajor_desc(bh + (uint32_t)j * 2 * UM_LBO);
                const uint64_t dbl = kmajor_desc(bl + (uint32_t)j * 2 * UM_LBO);
                const uint32_t first = (c % UM_SEG != 0 || j > 0) ? 1u : 0u;
                umma_ts(d, ta + 8u * j, dbh, idesc, first);
                umma_ts(d, ta + 8u * j, dbl, idesc, 1u);
                umma_ts(d, ta + UM_KC + 8u * j, dbh, idesc, 1u);
            }
            umma_commit(&empty[s]);
            if (c % UM_SEG == UM_SEG - 1 || c == C - 1) umma_commit(&acc_full[a]);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();  // every role has left its loop
    if (warp == UM_WARPS - 1 && lane == 0) {
        // products already issued (all of them, after a wait gave up) may still read the operand
        // stages and write tensor memory: the issuing thread waits for them, with the full bound,
        // before the CTA frees its memory
        umma_commit(&fin);
        mbar_wait(&fin, 0, UM_SPIN_FINAL);
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

bool i2o_umma_eligible(bool cplx, int precision, const DMap &m, int nq) {
    // from 4 FP32 columns (2 complex right-hand sides) the MMA tile (padded to N = 16) beats the
    // FP64 mma.sync tile path; a single right-hand side stays on the FMA tile path
    return precision == H2B_FP32 && m.coupling_kind == H2B_COUPLING_DENSE && (cplx ? 2 : 1) * nq >= 4;
}

cudaError_t launch_i2o_umma(bool cplx, const DMap &m, const DSide &recv, const DSide &src, const int *nodes,
                            int nnodes, const FarArgs &fa, int maxcoef, cudaStream_t st) {
    if (nnodes == 0) return cudaSuccess;
    const int nq = m.ncomp * fa.nrhs;
    const int ntmax = cplx ? UM_NT_MAX_CPLX : UM_NT_MAX_REAL;
    // right-hand sides per tile: at most ntmax, tiles of equal width
    const int ntiles = (nq + ntmax - 1) / ntmax;
    // a multiple of 8, so that the imaginary rows of a complex tile start on a 16-column boundary
    // of tensor memory; rows past the right-hand sides are zero
    const int qt_max = ((nq + ntiles - 1) / ntiles + 7) / 8 * 8;
    const int np = (((cplx ? 2 : 1) * qt_max + 15) / 16) * 16;
    // expanded moment stages (hi and lo), the raw moment ring and the coupling column stages
    const size_t eb = cplx ? 8 : 4, kq = cplx ? UM_KC / 2 : UM_KC;
    const size_t raw = ((size_t)UM_RS * qt_max * UM_RAWROW + 127) & ~(size_t)127;
    const size_t acols = (size_t)UM_AR * ((kq * maxcoef * eb + 127) & ~(size_t)127);
    size_t smem = (size_t)UM_NS * 2 * np * UM_KC * 4 + raw;
    // the coupling column stages grow with the block size; blocks whose stages do not fit beside
    // the moment stages are read by the register path instead
    int dev = 0, optin = 0;
    cudaError_t e0 = cudaGetDevice(&dev);
    if (e0 == cudaSuccess) e0 = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e0 != cudaSuccess) return e0;
    DMap mm = m;
    if (mm.cpl_vec && smem + acols + 1024 <= (size_t)optin)
        smem += acols;
    else
        mm.cpl_vec = 0;
    const dim3 grid(nnodes, (maxcoef + UM_M - 1) / UM_M, ntiles);
    auto go = [&](auto kern, auto *am, auto *dm) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, UM_THREADS, smem, st>>>(mm, recv, src, nodes, fa.mode, fa.nrhs, qt_max, am, dm);
        return cudaGetLastError();
    };
    if (cplx)
        return go(&i2o_umma_kernel<cfloat>, static_cast<const cfloat *>(fa.am), static_cast<cfloat *>(fa.dm));
    return go(&i2o_umma_kernel<float>, static_cast<const float *>(fa.am), static_cast<float *>(fa.dm));
}

cudaError_t read_umma_timeouts(unsigned *count) {
    return cudaMemcpyFromSymbol(count, g_umma_timeouts, sizeof(unsigned));
}

cudaError_t copy_umma_timeouts_async(unsigned *host, cudaStream_t st) {
    return cudaMemcpyFromSymbolAsync(host, g_umma_timeouts, sizeof(unsigned), 0, cudaMemcpyDeviceToHost, st);
}

cudaError_t set_umma_wait_limit(unsigned limit) {
    const unsigned v = limit ? limit : UM_SPIN;
    return cudaMemcpyToSymbol(g_umma_wait_limit, &v, sizeof(unsigned));
}

}  // namespace h2b
