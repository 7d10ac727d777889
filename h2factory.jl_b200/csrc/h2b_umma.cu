// B1 dense I2O of the FP32 form on the fifth-generation tensor cores (tcgen05, kind::tf32).
//
// Per receiving node r: l_r = sum over its pairs of op(B_pair) m_src (translateintonode!,
// src/farinteractions/traversalhelpers.jl:167-219, with the dense applycouplingkernel! of
// src/farinteractions/i2otranslations/i2otranslationcollection.jl:367-409 and the orientation rule
// of i2oprotocol.jl:87-92). For one receiver this is one GEMM whose K dimension runs over the
// concatenated pairs: D[nc x nq] = [op(B_1) op(B_2) ...] [m_1; m_2; ...].
//
// One CTA per (receiver, 128-row tile of its coefficients, tile of right-hand sides), two CTAs per
// SM. The K dimension streams in chunks of 16 FP32 values: every thread copies its share of chunk
// c + 3 from global memory (L2-resident couplings and moments) into a 4-stage ring of raw shared
// buffers with cp.async (gathers and zero fill included), so three chunks are in flight without
// registers; a split pass turns raw chunk c into the canonical no-swizzle K-major layout of the
// tensor cores, each FP32 value as a TF32 high part and a TF32 remainder; one thread issues per
// 8-wide k step the three products hi*hi + hi*lo + lo*hi (the lo*lo term is below FP32 rounding)
// into an FP32 accumulator in tensor memory, and a commit to an mbarrier per split buffer releases
// it, so splitting chunk c + 1 overlaps the products of chunk c. Accumulators live for 8 chunks (48
// MMAs) only: two alternate, and each finished one is added into an FP64 sum kept in tensor memory,
// because every MMA rounds its accumulator toward zero (one accumulator through a whole interaction
// list, ~30,000 MMAs, measured 1e-4 relative error; segments keep it near FP32 rounding). The
// epilogue reads the sums with tcgen05.ld and stores the FP32 moments.
//
// Complex maps run as real GEMMs: with B = Br + i Bi and m = mr + i mi,
//   [Re l | Im l] = [Br Bi] (interleaved along k) x [[mr, mi]; [-mi, mr]] (interleaved rows),
// so the coupling's interleaved (re, im) storage is the A operand as it lies in memory and each
// moment value feeds two B rows. Adjoint maps conjugate B in the split pass; symmetry-reduced
// couplings apply their row / column permutations in the copy addresses.
//
// Every wait on an mbarrier is bounded: a wait that gives up counts itself in a device counter
// (h2b_tensor_wait_timeouts), the CTA stops issuing, frees its tensor memory and returns.

#include "h2b_internal.cuh"

namespace h2b {

namespace {

constexpr int UM_M = 128;        // output rows per tile = tensor-memory lanes
constexpr int UM_KC = 16;        // FP32 K values per chunk: 4 groups of 16 bytes per row
constexpr int UM_KG = UM_KC / 4;
constexpr int UM_THREADS = 256;
constexpr int UM_NT_MAX = 64;    // MMA N (FP32 accumulator columns) per tile, at most
constexpr int UM_SEG = 8;        // chunks (48 MMAs) per accumulation segment
constexpr int UM_RS = 4;         // raw stages: chunks c + 1 .. c + 3 in flight while c is split
constexpr uint32_t UM_LBO = 128;           // bytes between the two 16-byte K halves of a k step
constexpr uint32_t UM_SBO = UM_KG * 128;   // bytes between 8-row groups (4 groups of 128 bytes)
constexpr uint32_t UM_AHALF = UM_M * UM_KC * 4;  // bytes of one A split part (8 KB)
constexpr uint32_t UM_RAWROW = UM_KC * 4 + 16;   // raw row layout: 64 bytes + 16 of padding
constexpr uint32_t UM_RAWA = UM_M * UM_RAWROW;   // raw A bytes (>= the column layouts' 8,448)
constexpr unsigned UM_SPIN = 1u << 22;           // try_wait attempts before a wait gives up
constexpr int UM_XMAP = 512;     // moment-row permutations up to this length are read from shared memory

__device__ unsigned int g_umma_timeouts = 0;

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

// v = hi + lo with hi, lo TF32: the high part and the rounded remainder
__device__ __forceinline__ void st_split(uint32_t hi_addr, uint32_t lo_addr, float a, float b, float c, float d) {
    const uint32_t h0 = tf32_bits(a), h1 = tf32_bits(b), h2 = tf32_bits(c), h3 = tf32_bits(d);
    const uint32_t l0 = tf32_bits(a - __uint_as_float(h0)), l1 = tf32_bits(b - __uint_as_float(h1));
    const uint32_t l2 = tf32_bits(c - __uint_as_float(h2)), l3 = tf32_bits(d - __uint_as_float(h3));
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(hi_addr), "r"(h0), "r"(h1), "r"(h2), "r"(h3));
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(lo_addr), "r"(l0), "r"(l1), "r"(l2), "r"(l3));
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
                 : "memory");
}

// bounded wait for the completion of the mbarrier phase with the given parity
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    const uint32_t a = su32(bar);
    for (unsigned it = 0; it < UM_SPIN; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    atomicAdd(&g_umma_timeouts, 1u);
    return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
        "%13, %14, %15, %16};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
        "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = __uint_as_float(r[u]);
}

// element copy global -> shared; src_bytes 0 writes zeros (src is then not read)
template <int EB>
__device__ __forceinline__ void cp_elem(uint32_t dst, const void *src, bool ok) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(dst), "l"(src), "n"(EB), "r"(ok ? EB : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_commit_group() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_wait_group() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <class T> struct UmScalar;
template <> struct UmScalar<float> {
    static constexpr int W = 1;  // FP32 values per element
};
template <> struct UmScalar<cfloat> {
    static constexpr int W = 2;
};

// The operands of one pair: op(B)[i, k] and the source moment rows, with the permutations of a
// symmetry-reduced coupling (sets [rowperm | rowperm^-1 | colperm | colperm^-1]) resolved.
template <class T>
struct UmPair {
    const T *B;   // coupling block
    const T *X;   // source moments, column-major snc x nq
    int snc;      // source coefficients
    int nk;       // K chunks
    const int *rowmap;  // output row -> row (forward) / column (transposed) of B, or null
    const int *xmap;    // k -> source moment row, or null
};

}  // namespace

template <class T>
__global__ void __launch_bounds__(UM_THREADS)
i2o_umma_kernel(DMap m, DSide r, DSide t, const int *__restrict__ nodes, int mode, int nrhs, int qt_max,
                const T *__restrict__ am, T *__restrict__ dm) {
    constexpr int W = UmScalar<T>::W;
    constexpr int EB = sizeof(T);        // bytes per element (4 real, 8 complex)
    constexpr int KQ = UM_KC / W;        // elements along k per chunk
    extern __shared__ __align__(128) unsigned char um_smem[];
    __shared__ uint64_t bar[2];
    __shared__ uint32_t tmem_slot;
    __shared__ int nchunks_s;
    __shared__ int xmap_s[UM_XMAP];  // the copied pair's moment-row permutation

    const int node = nodes[blockIdx.x];
    const int nc = um_ncoef(r, r.level[node]);
    const int m0 = blockIdx.y * UM_M;
    const int nq = m.ncomp * nrhs;
    const int q0 = blockIdx.z * qt_max;
    if (m0 >= nc || q0 >= nq) return;  // whole CTA, before any barrier
    const int mt = min(UM_M, nc - m0);
    const int qt = min(qt_max, nq - q0);
    const int nt = ((W * qt + 15) / 16) * 16;                 // MMA N of this tile
    const int ntmax = ((W * qt_max + 15) / 16) * 16;          // B rows a split buffer holds
    const int lb = W == 1 ? nt : ((qt + 7) / 8) * 8;          // B rows copied per chunk
    const int lbmax = W == 1 ? ntmax : ((qt_max + 7) / 8) * 8;
    const uint32_t split_bytes = 2 * UM_AHALF + 2u * (uint32_t)ntmax * (UM_KC * 4);
    const uint32_t raw_bytes = UM_RAWA + (uint32_t)lbmax * UM_RAWROW;
    const int p0 = r.i2o_ptr[node], p1 = r.i2o_ptr[node + 1];
    T *out = dm + r.mom_off[node] * nrhs;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (p0 == p1) {
        for (int o = tid; o < mt * qt; o += UM_THREADS) out[(int64_t)(q0 + o / mt) * nc + m0 + o % mt] = T{};
        return;
    }
    const bool fwd = mode == H2B_FORWARD, adj = mode == H2B_ADJOINT;
    const T *B0 = static_cast<const T *>(m.cpl);

    // tensor memory: two FP32 accumulators of ntmax columns (segments alternate between them) and
    // the FP64 sum of the drained segments (two columns per value), rounded up to a power of two
    const uint32_t ncols = ntmax <= 16 ? 64u : (ntmax <= 32 ? 128u : 256u);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_slot)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&bar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&bar[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        nchunks_s = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;

    auto pair_at = [&](int p) {
        UmPair<T> u;
        u.snc = um_ncoef(t, t.level[r.i2o_src[p]]);
        u.nk = (W * u.snc + UM_KC - 1) / UM_KC;
        u.B = B0 + r.pair_cpl[p];
        u.X = am + r.pair_src[p] * nrhs + (int64_t)q0 * u.snc;
        const int64_t ps = r.pair_perm ? r.pair_perm[p] : -1;
        u.rowmap = nullptr;
        u.xmap = nullptr;
        if (ps >= 0) {
            if (fwd) {  // t[rp[i], cp[j]] = M[i, j]: out[i] += sum_j M[rp^-1[i], j] x[cp[j]]
                u.rowmap = m.perm + ps + nc;
                u.xmap = m.perm + ps + 2 * nc;
            } else {    // out[j] += sum_i op(M)[cp^-1[j], i] x[rp[i]]
                u.rowmap = m.perm + ps + 3 * u.snc;
                u.xmap = m.perm + ps;
            }
        }
        return u;
    };
    {  // chunks of the whole interaction list
        int mine = 0;
        for (int p = p0 + tid; p < p1; p += UM_THREADS) mine += (W * um_ncoef(t, t.level[r.i2o_src[p]]) + UM_KC - 1) / UM_KC;
        if (mine) atomicAdd(&nchunks_s, mine);
        __syncthreads();
    }
    const int C = nchunks_s;

    // Copy mappings. A, forward blocks (column-major, rows contiguous): thread = one tile row,
    // consecutive lanes consecutive rows, raw layout [k][row]. A, transposed blocks (rows
    // contiguous along k) and B (moment columns contiguous along k): a warp covers 8 rows x 4
    // consecutive k, raw layout [row][k] with 80-byte rows. The tile rows a thread copies are
    // fixed, so a permuted block's row map is read once per pair.
    const int arow_f = tid & (UM_M - 1);                       // forward: the thread's row
    const int arow_t0 = (warp & 7) * 8 + (lane & 7);           // transposed: rows arow_t0, + 64
    const uint32_t colstride = UM_M * EB + 16;                 // raw column layout: bytes per k
    // copy cursor: pair pp, its chunk pk, chunks issued; the next pair's operands and row map are
    // fetched a pair ahead (their loads complete while the current pair streams), and a permuted
    // pair's moment-row map is staged in shared memory once per pair
    int pp = p0, pk = 0, issued = 0;
    UmPair<T> pu = pair_at(p0), pn = pu;
    int hrow[2], hrow_n[2];
    auto rows_of = [&](const UmPair<T> &u, int (&h)[2]) {
        if (fwd) {
            h[0] = arow_f < mt ? (u.rowmap ? u.rowmap[m0 + arow_f] : m0 + arow_f) : 0;
            h[1] = 0;
        } else {
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int rr = arow_t0 + 64 * e;
                h[e] = rr < mt ? (u.rowmap ? u.rowmap[m0 + rr] : m0 + rr) : 0;
            }
        }
    };
    auto fill_xmap = [&]() {  // every thread calls it (one barrier)
        if (pu.xmap && pu.snc <= UM_XMAP)
            for (int k = tid; k < pu.snc; k += UM_THREADS) xmap_s[k] = pu.xmap[k];
        __syncthreads();
    };
    rows_of(pu, hrow);
    if (p0 + 1 < p1) {
        pn = pair_at(p0 + 1);
        rows_of(pn, hrow_n);
    }
    fill_xmap();
    const uint32_t smem0 = su32(um_smem);
    const uint32_t raw0 = smem0 + 2 * split_bytes;
    auto issue = [&]() {  // copies of the next chunk into raw stage (issued % UM_RS); one group
        if (issued < C) {
            const uint32_t ra = raw0 + (uint32_t)(issued % UM_RS) * raw_bytes, rb = ra + UM_RAWA;
            const int kq0 = pk * KQ;
            if (fwd) {
#pragma unroll
                for (int j = 0; j < KQ / 2; ++j) {
                    const int kq = (tid >> 7) + 2 * j, k = kq0 + kq;
                    const bool ok = arow_f < mt && k < pu.snc;
                    cp_elem<EB>(ra + (uint32_t)kq * colstride + (uint32_t)arow_f * EB,
                                ok ? pu.B + hrow[0] + (int64_t)k * nc : pu.B, ok);
                }
            } else {
#pragma unroll
                for (int j = 0; j < KQ / 2; ++j) {
                    const int row = arow_t0 + 64 * (j & 1), kq = (j >> 1) * 4 + (lane >> 3), k = kq0 + kq;
                    const bool ok = row < mt && k < pu.snc;
                    cp_elem<EB>(ra + (uint32_t)row * UM_RAWROW + (uint32_t)kq * EB,
                                ok ? pu.B + k + (int64_t)hrow[j & 1] * pu.snc : pu.B, ok);
                }
            }
            const int nrb = lb >> 3;
            for (int e = tid; e < lb * KQ; e += UM_THREADS) {
                const int w = e >> 5, l = e & 31;
                const int q = (w % nrb) * 8 + (l & 7), kq = (w / nrb) * 4 + (l >> 3), k = kq0 + kq;
                const bool ok = q < qt && k < pu.snc;
                const T *src = pu.X;
                if (ok)
                    src = pu.X + (int64_t)q * pu.snc +
                          (pu.xmap ? (pu.snc <= UM_XMAP ? xmap_s[k] : pu.xmap[k]) : k);
                cp_elem<EB>(rb + (uint32_t)q * UM_RAWROW + (uint32_t)kq * EB, src, ok);
            }
            ++issued;
            if (++pk == pu.nk) {
                pk = 0;
                if (++pp < p1) {
                    pu = pn;
                    hrow[0] = hrow_n[0];
                    hrow[1] = hrow_n[1];
                    if (pp + 1 < p1) {
                        pn = pair_at(pp + 1);
                        rows_of(pn, hrow_n);
                    }
                    __syncthreads();  // every thread's copies read the previous pair's map
                    fill_xmap();
                }
            }
        }
        cp_commit_group();
    };
    // raw chunk -> split buffer: TF32 hi / lo in the canonical layout (A conjugated for adjoint maps)
    auto split = [&](uint32_t ra, uint32_t sbase) {
        const uint32_t rb = ra + UM_RAWA;
        const uint32_t ahi = sbase, alo = sbase + UM_AHALF;
        const uint32_t bhi = sbase + 2 * UM_AHALF, blo = bhi + (uint32_t)ntmax * (UM_KC * 4);
#pragma unroll
        for (int j = 0; j < UM_M * UM_KG / UM_THREADS; ++j) {
            const int g = tid + UM_THREADS * j;
            int row, kg;
            float v[4];
            if (fwd) {
                row = g & (UM_M - 1);
                kg = g >> 7;
                if constexpr (W == 1) {
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v[e]) : "r"(ra + (uint32_t)(4 * kg + e) * colstride + (uint32_t)row * 4));
                } else {
#pragma unroll
                    for (int e = 0; e < 2; ++e)
                        asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];"
                                     : "=f"(v[2 * e]), "=f"(v[2 * e + 1])
                                     : "r"(ra + (uint32_t)(2 * kg + e) * colstride + (uint32_t)row * 8));
                }
            } else {
                const int w = g >> 5, l = g & 31;
                row = (w & 15) * 8 + (l & 7);
                kg = (w >> 4) * 4 + (l >> 3);
                asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                             : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3])
                             : "r"(ra + (uint32_t)row * UM_RAWROW + (uint32_t)kg * 16));
            }
            if (W == 2 && adj) {
                v[1] = -v[1];
                v[3] = -v[3];
            }
            const uint32_t o = goff(row, kg);
            st_split(ahi + o, alo + o, v[0], v[1], v[2], v[3]);
        }
        for (int g = tid; g < lb * UM_KG; g += UM_THREADS) {
            const int q = g >> 2, kg = g & 3;
            float v[4];
            asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                         : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3])
                         : "r"(rb + (uint32_t)q * UM_RAWROW + (uint32_t)kg * 16));
            if constexpr (W == 1) {
                const uint32_t o = goff(q, kg);
                st_split(bhi + o, blo + o, v[0], v[1], v[2], v[3]);
            } else if (q < qt) {
                // row q: (mr, -mi) per k feeds Re; row qt + q: (mi, mr) feeds Im
                const uint32_t o1 = goff(q, kg), o2 = goff(qt + q, kg);
                st_split(bhi + o1, blo + o1, v[0], -v[1], v[2], -v[3]);
                st_split(bhi + o2, blo + o2, v[1], v[0], v[3], v[2]);
            }
        }
    };

    // The tensor cores round each MMA's sum toward zero, so one FP32 accumulator carried through
    // thousands of MMAs loses ~1e-4 of its value. Chunks are therefore summed in segments of
    // UM_SEG chunks, alternating between two accumulators; each finished segment is added into an
    // FP64 running sum in tensor memory while the next one is on the tensor cores.
    const int lq = warp & 3, half = warp >> 2;  // warp w reads lanes 32 (w % 4) .. + 31
    const int row = 32 * lq + lane;
    const uint32_t tlane = tmem + ((uint32_t)(32 * lq) << 16);
    const uint32_t tmaster = tlane + 2u * (uint32_t)ntmax;
    auto drain = [&](int a, bool first) {  // master (+)= accumulator a, over this warp's half
        const int hw = ntmax / 2;
        for (int j0 = half * hw; j0 < (half + 1) * hw && j0 < nt; j0 += 8) {
            float v[8];
            tmem_ld8(tlane + (uint32_t)(a * ntmax + j0), v);
            uint32_t w[16];
            if (!first) tmem_ld16(tmaster + 2u * (uint32_t)j0, w);
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const double mv = (first ? 0.0 : __hiloint2double((int)w[2 * u + 1], (int)w[2 * u])) + (double)v[u];
                w[2 * u] = (uint32_t)__double2loint(mv);
                w[2 * u + 1] = (uint32_t)__double2hiint(mv);
            }
            tmem_st16(tmaster + 2u * (uint32_t)j0, w);
        }
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    };

    const uint32_t idesc = tf32_idesc(UM_M, nt);
#pragma unroll
    for (int s = 0; s < UM_RS - 1; ++s) issue();
    int c = 0;
    bool bad = false;
    for (; c < C; ++c) {
        const int s = c & 1, g = c / UM_SEG, a = g & 1;
        const uint32_t sbase = smem0 + (uint32_t)s * split_bytes;
        cp_wait_group<UM_RS - 2>();  // this thread's copies of chunk c have landed
        __syncthreads();             // everyone's have
        // the products of chunk c - 2 read this split buffer: wait for their commit
        if (c >= 2 && !bad) bad = !mbar_wait(&bar[s], ((c - 2) >> 1) & 1);
        if (c % UM_SEG == 0 && g >= 2) {
            // segment g - 2 ended at chunk (g - 1) UM_SEG - 1 <= c - 2: complete; free its
            // accumulator for segment g
            if (__syncthreads_or(bad)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            drain(a, g == 2);
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        }
        if (!bad) split(raw0 + (uint32_t)(c % UM_RS) * raw_bytes, sbase);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if (__syncthreads_or(bad)) break;
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t dacc = tmem + (uint32_t)(a * ntmax);
            const uint32_t ahi = sbase, alo = sbase + UM_AHALF;
            const uint32_t bhi = sbase + 2 * UM_AHALF, blo = bhi + (uint32_t)ntmax * (UM_KC * 4);
#pragma unroll
            for (int j = 0; j < UM_KC / 8; ++j) {
                const uint32_t k = (uint32_t)j * 2 * UM_LBO;
                umma_tf32(dacc, kmajor_desc(ahi + k), kmajor_desc(bhi + k), idesc,
                          (c % UM_SEG != 0 || j > 0) ? 1u : 0u);
                umma_tf32(dacc, kmajor_desc(ahi + k), kmajor_desc(blo + k), idesc, 1u);
                umma_tf32(dacc, kmajor_desc(alo + k), kmajor_desc(bhi + k), idesc, 1u);
            }
            umma_commit(&bar[s]);
        }
        issue();  // chunk c + UM_RS - 1 into the raw stage chunk c - 1 used
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    // the last commit completes after every product issued before it
    if (!bad && c > 0) bad = !mbar_wait(&bar[(c - 1) & 1], ((c - 1) >> 1) & 1);
    bad = __syncthreads_or(bad);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!bad) {
        // total = FP64 sum of segments 0 .. G-3 + accumulators of segments G-2 and G-1; warps w
        // and w + 4 take alternate blocks of 8 right-hand sides
        const int G = (c + UM_SEG - 1) / UM_SEG;
        auto total8 = [&](int col, double (&v)[8]) {
            float f[8];
            tmem_ld8(tlane + (uint32_t)(((G - 1) & 1) * ntmax + col), f);
#pragma unroll
            for (int u = 0; u < 8; ++u) v[u] = f[u];
            if (G >= 2) {
                tmem_ld8(tlane + (uint32_t)(((G - 2) & 1) * ntmax + col), f);
#pragma unroll
                for (int u = 0; u < 8; ++u) v[u] += f[u];
            }
            if (G >= 3) {
                uint32_t w[16];
                tmem_ld16(tmaster + 2u * (uint32_t)col, w);
#pragma unroll
                for (int u = 0; u < 8; ++u) v[u] += __hiloint2double((int)w[2 * u + 1], (int)w[2 * u]);
            }
        };
        for (int j8 = half; j8 * 8 < qt; j8 += 2) {
            double re[8];
            total8(8 * j8, re);
            if constexpr (W == 1) {
                if (row < mt) {
#pragma unroll
                    for (int u = 0; u < 8; ++u)
                        if (8 * j8 + u < qt) out[(int64_t)(q0 + 8 * j8 + u) * nc + m0 + row] = (float)re[u];
                }
            } else {
                double im[8];
                total8(qt + 8 * j8, im);
                if (row < mt) {
#pragma unroll
                    for (int u = 0; u < 8; ++u)
                        if (8 * j8 + u < qt)
                            out[(int64_t)(q0 + 8 * j8 + u) * nc + m0 + row] = T{(float)re[u], (float)im[u]};
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

bool i2o_umma_eligible(bool cplx, int precision, const DMap &m, int nq) {
    // from 4 FP32 columns (2 complex right-hand sides) the MMA tile (padded to N = 16) beats the
    // FP64 mma.sync tile path (sphere shape at 32,768 points, 2-4 complex RHS: 16.2 vs 20.5 ms per
    // product); a single right-hand side stays on the FMA tile path (11.9 vs 14.7 ms)
    return precision == H2B_FP32 && m.coupling_kind == H2B_COUPLING_DENSE && (cplx ? 2 : 1) * nq >= 4;
}

cudaError_t launch_i2o_umma(bool cplx, const DMap &m, const DSide &recv, const DSide &src, const int *nodes,
                            int nnodes, const FarArgs &fa, int maxcoef, cudaStream_t st) {
    if (nnodes == 0) return cudaSuccess;
    const int W = cplx ? 2 : 1;
    const int nq = m.ncomp * fa.nrhs;
    // right-hand sides per tile: MMA N = W * qt <= 64, tiles of equal width
    const int ntiles = (W * nq + UM_NT_MAX - 1) / UM_NT_MAX;
    const int qt_max = (nq + ntiles - 1) / ntiles;
    const int ntmax = ((W * qt_max + 15) / 16) * 16;
    const int lbmax = cplx ? ((qt_max + 7) / 8) * 8 : ntmax;
    // two split buffers (A and B, TF32 hi and lo) and UM_RS raw stages
    const size_t smem = 2 * (2 * (size_t)UM_AHALF + 2 * (size_t)ntmax * (UM_KC * 4)) +
                        (size_t)UM_RS * (UM_RAWA + (size_t)lbmax * UM_RAWROW);
    const dim3 grid(nnodes, (maxcoef + UM_M - 1) / UM_M, ntiles);
    auto go = [&](auto kern, auto *am, auto *dm) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, UM_THREADS, smem, st>>>(m, recv, src, nodes, fa.mode, fa.nrhs, qt_max, am, dm);
        return cudaGetLastError();
    };
    if (cplx)
        return go(&i2o_umma_kernel<cfloat>, static_cast<const cfloat *>(fa.am), static_cast<cfloat *>(fa.dm));
    return go(&i2o_umma_kernel<float>, static_cast<const float *>(fa.am), static_cast<float *>(fa.dm));
}

cudaError_t read_umma_timeouts(unsigned *count) {
    return cudaMemcpyFromSymbol(count, g_umma_timeouts, sizeof(unsigned));
}

}  // namespace h2b
