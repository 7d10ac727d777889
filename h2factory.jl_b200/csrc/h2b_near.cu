// Near field (nearmul!, src/nearinteractions/nearmul.jl:8-14) on sm_100a.
//
// Layout in HBM: every dense block of a (output leaf, input leaf) pair is stored column-major with
// an even leading dimension for real fields, so that each lane of a warp streams two consecutive
// rows with one 16-byte load. The blocks of one output leaf are split across the warps of one CTA;
// every warp sweeps its blocks column by column with x broadcast from shared memory, and
// the warps' partial rows are summed in shared memory at the end. Transposed and adjoint products
// run the same kernel on the transposed operator: N itself when N^T == N (checked once on the
// device when the core is built), otherwise a transposed copy of the blocks built at upload.

#include <algorithm>
#include <type_traits>

#include "h2b_internal.cuh"

namespace h2b {

namespace {

constexpr int NEAR_WARPS = 8;

template <class V> struct NearVec;
template <> struct NearVec<double> {
    static constexpr int RPL = 2;  // rows per lane per load
};
template <> struct NearVec<cdouble> {
    static constexpr int RPL = 1;
};

// streaming (evict-first) loads of the near blocks: they are read once per product
__device__ __forceinline__ void load_rows(const double *p, double (&v)[2]) {
    const double2 t = __ldcs(reinterpret_cast<const double2 *>(p));
    v[0] = t.x;
    v[1] = t.y;
}
__device__ __forceinline__ void load_rows(const cdouble *p, cdouble (&v)[1]) {
    const double2 t = __ldcs(reinterpret_cast<const double2 *>(p));
    v[0] = {t.x, t.y};
}

__device__ __forceinline__ double fma_c(double a, double b, double c, bool) { return fma(a, b, c); }
__device__ __forceinline__ cdouble fma_c(cdouble a, cdouble b, cdouble c, bool cjg) {
    // c + op(a) * b, op = conj when cjg
    const double ay = cjg ? -a.y : a.y;
    return {fma(a.x, b.x, fma(-ay, b.y, c.x)), fma(a.x, b.y, fma(ay, b.x, c.y))};
}

// R x values of one column from shared memory, two per 16-byte load where the type allows
template <class V, int R>
__device__ __forceinline__ void load_x(const V *p, V (&v)[R]) {
    if constexpr (sizeof(V) == 8 && R % 2 == 0) {
#pragma unroll
        for (int q = 0; q < R; q += 2) {
            const double2 t = *reinterpret_cast<const double2 *>(p + q);
            v[q] = t.x;
            v[q + 1] = t.y;
        }
    } else {
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = p[q];
    }
}

__device__ __forceinline__ int near_ld(int nr, double *) { return nr + (nr & 1); }
__device__ __forceinline__ int near_ld(int nr, cdouble *) { return nr; }

// y[rows(g)] = alpha * op(N_g) x + beta * y[rows(g)] for right-hand sides [r0, r0 + R).
// A pass covers MP chunks of 32 * RPL rows, so a leaf of up to 32 * RPL * MP rows takes a single
// sweep over its blocks (one x gather per column chunk, no column split between passes). UB
// columns are loaded before any is used.
// Shared memory: per warp, the x values of its current 32-column chunk ([32][R]), read back as
// broadcasts; then the warps' partial rows ([NEAR_WARPS][RPP][R]) for the final reduction.
template <class V, int R, int MP, int UB, int MINB>
__global__ void __launch_bounds__(NEAR_WARPS * 32, MINB)
near_rows_kernel(NearOp op, DSide outs, DSide ins, bool cjg, int r0, int rc, const V *__restrict__ x,
                 int64_t ldx, V *__restrict__ y, int64_t ldy, V alpha, V beta, bool beta_zero) {
    constexpr int RPL = NearVec<V>::RPL;
    constexpr int RPC = 32 * RPL;  // rows per chunk
    constexpr int RPP = RPC * MP;  // rows per pass
    extern __shared__ unsigned char smem_raw[];
    const int g = blockIdx.x;
    const int leaf = op.grp_leaf[g];
    const int o0 = outs.value_ptr[leaf], nr = outs.value_ptr[leaf + 1] - o0;
    const int u0 = op.unit_ptr[g], u1 = op.unit_ptr[g + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    V *xs = reinterpret_cast<V *>(smem_raw) + warp * 32 * R;                 // this warp's x chunk
    V *part = reinterpret_cast<V *>(smem_raw) + NEAR_WARPS * 32 * R;         // partial rows
    const V *D = static_cast<const V *>(op.data);
    const int ld = near_ld(nr, (V *)nullptr);
    for (int p0 = 0; p0 < nr; p0 += RPP) {
        const int i0 = p0 + RPL * lane;  // first row of this lane in chunk 0
        bool live[MP];                   // lanes past the last row load nothing
        bool any[MP];                    // warp-uniform: the chunk has rows at all
#pragma unroll
        for (int c = 0; c < MP; ++c) {
            live[c] = i0 + c * RPC < nr;
            any[c] = p0 + c * RPC < nr;
        }
        V acc[MP][RPL][R];
#pragma unroll
        for (int c = 0; c < MP; ++c)
#pragma unroll
            for (int k = 0; k < RPL; ++k)
#pragma unroll
                for (int q = 0; q < R; ++q) acc[c][k][q] = V{};
        // work units are (block, 32-column chunk) pairs, dealt round-robin to the warps
        {
            for (int un = u0 + warp; un < u1; un += NEAR_WARPS) {
                const int4 ue = op.unit[un];
                const int jn = ue.y;
                __syncwarp();
                {
                    const int dof = lane < jn ? ins.value[ue.x + lane] : 0;
#pragma unroll
                    for (int q = 0; q < R; ++q)
                        xs[lane * R + q] = (lane < jn && q < rc) ? x[(int64_t)(r0 + q) * ldx + dof] : V{};
                }
                __syncwarp();
                const V *Bj = D + (((int64_t)ue.w << 32) | (uint32_t)ue.z) + i0;
                int jj = 0;
                for (; jj + UB <= jn; jj += UB) {
                    V bv[UB][MP][RPL];  // UB columns in flight before any use
#pragma unroll
                    for (int u = 0; u < UB; ++u)
#pragma unroll
                        for (int c = 0; c < MP; ++c) {
                            if (live[c]) {
                                load_rows(Bj + (int64_t)(jj + u) * ld + c * RPC, bv[u][c]);
                            } else {
#pragma unroll
                                for (int k = 0; k < RPL; ++k) bv[u][c][k] = V{};
                            }
                        }
#pragma unroll
                    for (int u = 0; u < UB; ++u) {
                        V xv[R];
                        load_x<V, R>(xs + (jj + u) * R, xv);
#pragma unroll
                        for (int c = 0; c < MP; ++c) {
                            if (!any[c]) continue;
#pragma unroll
                            for (int q = 0; q < R; ++q)
#pragma unroll
                                for (int k = 0; k < RPL; ++k)
                                    acc[c][k][q] = fma_c(bv[u][c][k], xv[q], acc[c][k][q], cjg);
                        }
                    }
                }
                for (; jj < jn; ++jj) {
#pragma unroll
                    for (int c = 0; c < MP; ++c) {
                        if (!any[c]) continue;
                        V bv[RPL];
                        if (live[c]) {
                            load_rows(Bj + (int64_t)jj * ld + c * RPC, bv);
                        } else {
#pragma unroll
                            for (int k = 0; k < RPL; ++k) bv[k] = V{};
                        }
#pragma unroll
                        for (int q = 0; q < R; ++q) {
                            const V xv = xs[jj * R + q];
#pragma unroll
                            for (int k = 0; k < RPL; ++k) acc[c][k][q] = fma_c(bv[k], xv, acc[c][k][q], cjg);
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int c = 0; c < MP; ++c)
#pragma unroll
            for (int k = 0; k < RPL; ++k)
#pragma unroll
                for (int q = 0; q < R; ++q) part[(warp * RPP + c * RPC + RPL * lane + k) * R + q] = acc[c][k][q];
        __syncthreads();
        const int rows = min(RPP, nr - p0);
        for (int e = threadIdx.x; e < rows * rc; e += blockDim.x) {
            const int i = e / rc, q = e % rc;
            V s = V{};
#pragma unroll
            for (int w = 0; w < NEAR_WARPS; ++w) s = s + part[(w * RPP + i) * R + q];
            V *o = &y[(int64_t)(r0 + q) * ldy + outs.value[o0 + p0 + i]];
            const V v = alpha * s;
            *o = beta_zero ? v : v + beta * *o;
        }
        __syncthreads();
    }
}

// FP64 tensor-core MMA, m8n8k4 (PTX ISA fragment layout for .f64: A[lane/4][lane%4],
// B[lane%4][lane/4], C[lane/4][2*(lane%4) + i]).
__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// Gather for the tensor-core kernel below: the right-hand sides of input dof value[pos] as one
// contiguous row, xp[pos * R + q] = x[(r0 + q) * ldx + value[pos]] (zero for q >= rc), so a warp
// reads its 32-column x chunk as one 4 KB range instead of 512 scattered elements.
template <int R>
__global__ void near_gather_kernel(const int *__restrict__ value, int nvals, int r0, int rc,
                                   const double *__restrict__ x, int64_t ldx, double *__restrict__ xp) {
    const int64_t total = (int64_t)nvals * R;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int pos = (int)(e / R), q = (int)(e % R);
        xp[e] = q < rc ? x[(int64_t)(r0 + q) * ldx + value[pos]] : 0.0;
    }
}

// Real near blocks, 8 or 16 right-hand sides, on the FP64 tensor cores. Warps 0-3 take the
// first 32 rows of a 64-row pass and warps 4-7 the next 32; the (block, 32-column) units of the
// leaf are dealt round-robin to the 4 warps of each half. A warp streams its units through a
// private ring of MST stages in shared memory with cp.async (MCOLS columns of its 32-row slab and
// their gathered x rows per stage, near_gather_kernel), MST - 1 stages ahead of the one its MMAs
// consume, so HBM loads stay in flight without registers and no block-wide barrier runs until the
// partial rows meet (summed over the 4 warps of a half, in shared memory reusing the rings).
// Fragment row g of row tile t is slab row 4g + t, so a lane reads its 4 rows with two 16-byte
// loads. Rows and columns past the block are zero-filled by the copies (source size 0). Waits are
// on the warp's own copies (cp.async.wait_group, then __syncwarp). On the benchmark map this form
// is 4 % faster per served step than the same tiling with register-staged loads. Two stages per
// warp keep the CTA at 59 KB of shared memory and 78 registers, so three CTAs (24 warps) share an
// SM: 11 % faster for 16 right-hand sides than three stages at two CTAs per SM (837 vs 941 us on
// the benchmark map); four CTAs of 4-column stages spill and measured slower.
constexpr int MST = 2;                 // stages per warp
constexpr int MCOLS = 8;               // columns per stage
constexpr int MSA = 34;                // slab column stride (doubles): 16-byte fragment reads hit
                                       // the banks 4 lanes each, the minimum for 512 bytes

__device__ __forceinline__ void cp16(void *smem, const void *gmem, bool valid) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <int NT>
constexpr size_t mma_pipe_smem() {  // all warps' rings (also holds the partial rows afterwards)
    return (size_t)NEAR_WARPS * MST * MCOLS * (MSA + 8 * NT + 8) * sizeof(double);
}

template <int NT>
__global__ void __launch_bounds__(NEAR_WARPS * 32, 3)
near_rows_mma_kernel(NearOp op, DSide outs, DSide ins, int r0, int rc, const double *__restrict__ xp,
                          double *__restrict__ y, int64_t ldy, double alpha, double beta, bool beta_zero) {
    constexpr int R = 8 * NT;
    constexpr int XS = R + 8;  // x row stride, 8 mod 16 doubles: two wavefronts per fragment read
    constexpr int SA = MCOLS * MSA, SX = MCOLS * XS, SS = SA + SX;  // doubles per stage
    static_assert(NEAR_WARPS * 32 * R <= NEAR_WARPS * MST * SS, "partial rows fit the rings");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int g = blockIdx.x;
    const int leaf = op.grp_leaf[g];
    const int o0 = outs.value_ptr[leaf], nr = outs.value_ptr[leaf + 1] - o0;
    const int u0 = op.unit_ptr[g], u1 = op.unit_ptr[g + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g4 = lane >> 2, t4 = lane & 3;
    const int half = warp >> 2, wq = warp & 3;
    double *ring = reinterpret_cast<double *>(smem_raw) + (size_t)warp * MST * SS;
    double *part = reinterpret_cast<double *>(smem_raw);  // [8 warps][32 rows][R], after the units
    const double *D = static_cast<const double *>(op.data);
    for (int p0 = 0; p0 < nr; p0 += 64) {
        const int rows0 = p0 + 32 * half;
        const bool active = rows0 < nr;
        const int rpairs = active ? (min(32, nr - rows0) + 1) / 2 : 0;  // 16-byte row pairs
        const int ld = nr + (nr & 1);
        // producer cursor: this warp's unit pu (units wq, wq + 4, ... of the group), its entry ue,
        // the next one un (loaded a unit ahead), and the first column pj of the next stage
        int pu = active ? u0 + wq : u1, pj = 0;
        int4 ue = pu < u1 ? op.unit[pu] : make_int4(0, 0, 0, 0);
        int4 un = pu + 4 < u1 ? op.unit[pu + 4] : ue;
        auto issue = [&](int slot) -> int {  // one commit group per call; 1 if it holds a stage
            int got = 0;
            if (pu < u1) {
                const int c0 = ue.x, nc = ue.y;
                const double *B = D + (((int64_t)ue.w << 32) | (uint32_t)ue.z) + rows0;
                double *sa = ring + slot * SS, *sx = sa + SA;
                // slab: MCOLS columns x 16 row pairs, 16-byte pieces
                for (int c = lane; c < MCOLS * 16; c += 32) {
                    const int col = c >> 4, rp = c & 15;
                    const bool ok = pj + col < nc && rp < rpairs;
                    cp16(sa + col * MSA + 2 * rp, ok ? B + (int64_t)(pj + col) * ld + 2 * rp : B, ok);
                }
                // x rows: MCOLS columns x R / 2 pieces
                for (int c = lane; c < MCOLS * R / 2; c += 32) {
                    const int col = c / (R / 2), q = 2 * (c % (R / 2));
                    const bool ok = pj + col < nc;
                    cp16(sx + col * XS + q, ok ? xp + (int64_t)(c0 + pj + col) * R + q : xp, ok);
                }
                got = 1;
                pj += MCOLS;
                if (pj >= nc) {
                    pj = 0;
                    pu += 4;
                    ue = un;
                    if (pu + 4 < u1) un = op.unit[pu + 4];
                }
            }
            cp_commit();
            return got;
        };
        double acc[4][NT][2];
#pragma unroll
        for (int t = 0; t < 4; ++t)
#pragma unroll
            for (int u = 0; u < NT; ++u) acc[t][u][0] = acc[t][u][1] = 0.0;
        int nstages = 0;  // stages issued so far; the loop below runs until it has consumed them all
#pragma unroll
        for (int s2 = 0; s2 < MST - 1; ++s2) nstages += issue(s2);
        int slot = 0;
        for (int st = 0; st < nstages; ++st) {
            nstages += issue((slot + MST - 1) % MST);
            cp_wait<MST - 1>();
            __syncwarp();
            const double *sa = ring + slot * SS + 4 * g4, *sx = ring + slot * SS + SA + g4;
#pragma unroll
            for (int kk = 0; kk < MCOLS; kk += 4) {
                const double2 a01 = *reinterpret_cast<const double2 *>(sa + (kk + t4) * MSA);
                const double2 a23 = *reinterpret_cast<const double2 *>(sa + (kk + t4) * MSA + 2);
                const double a[4] = {a01.x, a01.y, a23.x, a23.y};
                double b[NT];
#pragma unroll
                for (int u = 0; u < NT; ++u) b[u] = sx[(kk + t4) * XS + 8 * u];
#pragma unroll
                for (int t = 0; t < 4; ++t)
#pragma unroll
                    for (int u = 0; u < NT; ++u) dmma(acc[t][u], a[t], b[u]);
            }
            __syncwarp();  // the slot is read; the next issue may refill it
            slot = slot + 1 == MST ? 0 : slot + 1;
        }
        cp_wait<0>();
        __syncthreads();  // every warp is done with its ring: reuse it for the partial rows
#pragma unroll
        for (int t = 0; t < 4; ++t)
#pragma unroll
            for (int u = 0; u < NT; ++u)
#pragma unroll
                for (int h = 0; h < 2; ++h)
                    part[(warp * 32 + 4 * g4 + t) * R + 8 * u + 2 * t4 + h] = acc[t][u][h];
        __syncthreads();
        const int rows = min(64, nr - p0);
        for (int e = threadIdx.x; e < rows * rc; e += blockDim.x) {
            const int i = e / rc, q = e % rc;
            const int hf = i >> 5, li = i & 31;
            double sum = 0.0;
#pragma unroll
            for (int w = 0; w < 4; ++w) sum += part[((hf * 4 + w) * 32 + li) * R + q];
            double *o = &y[(int64_t)(r0 + q) * ldy + outs.value[o0 + p0 + i]];
            const double v = alpha * sum;
            *o = beta_zero ? v : v + beta * *o;
        }
        __syncthreads();
    }
}

template <int NT>
cudaError_t launch_rows_mma(const NearOp &op, const DSide &outs, const DSide &ins, int r0, int rc,
                                 const double *x, int64_t ldx, double *xp, double *y, int64_t ldy, double alpha,
                                 double beta, bool bz, cudaStream_t st) {
    constexpr int R = 8 * NT;
    const int nvals = ins.nvalues;
    near_gather_kernel<R><<<std::max(1, std::min(148 * 8, (int)(((int64_t)nvals * R + 255) / 256))), 256, 0, st>>>(
        ins.value, nvals, r0, rc, x, ldx, xp);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const size_t sm = mma_pipe_smem<NT>();
    e = cudaFuncSetAttribute(near_rows_mma_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    near_rows_mma_kernel<NT><<<op.ngroups, NEAR_WARPS * 32, sm, st>>>(op, outs, ins, r0, rc, xp, y, ldy,
                                                                           alpha, beta, bz);
    return cudaGetLastError();
}



// Complex near blocks, 8 or more right-hand sides, on the FP64 tensor cores. One warp (one CTA)
// per (output leaf, 32-row slab) work item (NearOp::slab): the warp streams the slab's rows of
// every block of the leaf through a private CST-stage cp.async ring (CCOLS columns and their
// gathered x rows per stage, zero-filled past the block) and keeps all R right-hand sides of its
// 32 rows in registers, so no partial rows are exchanged between warps and the block scheduler
// balances the items. A complex product runs as a real one without rearranging the stored block:
// its column k read as the two real columns (re, im) is the A operand along k' = 2k, 2k + 1, and
// with B rows [xr, xi] and [-xi, xr] (adjoint: [xi, -xr]) the real output columns are [Re y | Im y]:
//   Re y = sum_k ar xr - ai xi,  Im y = sum_k ar xi + ai xr.
// Fragment row g of row tile t is slab row 4g + t (m8n8k4: A[lane/4][lane%4], B[lane%4][lane/4]).
constexpr int CST = 3;     // ring stages per warp
constexpr int CCOLS = 4;   // complex columns per stage: two k steps
constexpr int CSA = 33;    // slab column stride in complex elements (32 rows + 1 of padding)

template <int R>
__global__ void __launch_bounds__(32, 16)
near_slab_mma_c_kernel(NearOp op, DSide outs, int r0, int rc, const cdouble *__restrict__ xp,
                       cdouble *__restrict__ y, int64_t ldy, cdouble alpha, cdouble beta, bool beta_zero,
                       bool cjg) {
    constexpr int NU = R / 8;                        // n tiles per block of R real columns
    constexpr int XS = R + 1;                        // x row stride (complex)
    constexpr int SS = CCOLS * CSA + CCOLS * XS;     // complex elements per stage
    __shared__ __align__(16) cdouble ring[CST * SS];
    const int2 item = op.slab[blockIdx.x];
    const int g = item.x, rows0 = 32 * item.y;
    const int leaf = op.grp_leaf[g];
    const int o0 = outs.value_ptr[leaf], nr = outs.value_ptr[leaf + 1] - o0;
    const int nrows = min(32, nr - rows0);
    const int u0 = op.unit_ptr[g], u1 = op.unit_ptr[g + 1];
    const int lane = threadIdx.x, g4 = lane >> 2, t4 = lane & 3;
    const cdouble *D = static_cast<const cdouble *>(op.data);
    // producer cursor: unit pu, its entry ue, first column pj of the next stage
    int pu = u0, pj = 0;
    int4 ue = pu < u1 ? op.unit[pu] : make_int4(0, 0, 0, 0);
    auto issue = [&](int slot) -> int {  // one commit group per call; 1 if it holds a stage
        int got = 0;
        if (pu < u1) {
            const int c0 = ue.x, nc = ue.y;
            const cdouble *B = D + (((int64_t)ue.w << 32) | (uint32_t)ue.z) + rows0;
            cdouble *sa = ring + slot * SS, *sx = sa + CCOLS * CSA;
#pragma unroll
            for (int col = 0; col < CCOLS; ++col) {
                const bool ok = pj + col < nc && lane < nrows;
                cp16(sa + col * CSA + lane, ok ? B + (int64_t)(pj + col) * nr + lane : B, ok);
            }
#pragma unroll
            for (int c = lane; c < CCOLS * R; c += 32) {
                const int col = c / R, q = c % R;
                const bool ok = pj + col < nc;
                cp16(sx + col * XS + q, ok ? xp + (int64_t)(c0 + pj + col) * R + q : xp, ok);
            }
            got = 1;
            pj += CCOLS;
            if (pj >= nc) {
                pj = 0;
                if (++pu < u1) ue = op.unit[pu];
            }
        }
        cp_commit();
        return got;
    };
    double acc[4][2 * NU][2];
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int u = 0; u < 2 * NU; ++u) acc[t][u][0] = acc[t][u][1] = 0.0;
    int nst = 0;
#pragma unroll
    for (int s2 = 0; s2 < CST - 1; ++s2) nst += issue(s2);
    int slot = 0;
    const int part = t4 & 1;
    for (int st = 0; st < nst; ++st) {
        nst += issue((slot + CST - 1) % CST);
        cp_wait<CST - 1>();
        __syncwarp();
        const double *sa = reinterpret_cast<const double *>(ring + slot * SS);
        const cdouble *sx = ring + slot * SS + CCOLS * CSA;
#pragma unroll
        for (int kk = 0; kk < CCOLS / 2; ++kk) {
            const int col = 2 * kk + (t4 >> 1);
            double a[4], b[2 * NU];
#pragma unroll
            for (int t = 0; t < 4; ++t) a[t] = sa[2 * (col * CSA + 4 * g4 + t) + part];
#pragma unroll
            for (int u = 0; u < NU; ++u) {
                const double2 xv = *reinterpret_cast<const double2 *>(sx + col * XS + 8 * u + g4);
                if (part == 0) {
                    b[u] = xv.x;
                    b[NU + u] = xv.y;
                } else {
                    b[u] = cjg ? xv.y : -xv.y;
                    b[NU + u] = cjg ? -xv.x : xv.x;
                }
            }
#pragma unroll
            for (int t = 0; t < 4; ++t)
#pragma unroll
                for (int u = 0; u < 2 * NU; ++u) dmma(acc[t][u], a[t], b[u]);
        }
        __syncwarp();  // the slot is read; the next issue may refill it
        slot = slot + 1 == CST ? 0 : slot + 1;
    }
    cp_wait<0>();
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const int row = 4 * g4 + t;
        if (row >= nrows) continue;
        const int64_t dof = outs.value[o0 + rows0 + row];
#pragma unroll
        for (int u = 0; u < NU; ++u)
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int q = 8 * u + 2 * t4 + i;
                if (q >= rc) continue;
                cdouble *o = &y[(int64_t)(r0 + q) * ldy + dof];
                const cdouble v = alpha * cdouble{acc[t][u][i], acc[t][NU + u][i]};
                *o = beta_zero ? v : v + beta * *o;
            }
    }
}

// complex x rows gathered in leaf order: xp[pos * R + q] = x[(r0 + q) * ldx + value[pos]]
template <int R>
__global__ void near_gather_c_kernel(const int *__restrict__ value, int nvals, int r0, int rc,
                                     const cdouble *__restrict__ x, int64_t ldx, cdouble *__restrict__ xp) {
    const int64_t total = (int64_t)nvals * R;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int pos = (int)(e / R), q = (int)(e % R);
        xp[e] = q < rc ? x[(int64_t)(r0 + q) * ldx + value[pos]] : cdouble{0.0, 0.0};
    }
}

template <int R>
cudaError_t launch_slab_mma_c(const NearOp &op, const DSide &outs, const DSide &ins, bool cjg, int r0, int rc,
                              const cdouble *x, int64_t ldx, cdouble *xp, cdouble *y, int64_t ldy, cdouble alpha,
                              cdouble beta, bool bz, cudaStream_t st) {
    const int nvals = ins.nvalues;
    near_gather_c_kernel<R><<<std::max(1, std::min(148 * 8, (int)(((int64_t)nvals * R + 255) / 256))), 256, 0, st>>>(
        ins.value, nvals, r0, rc, x, ldx, xp);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || op.nslabs == 0) return e;
    near_slab_mma_c_kernel<R><<<op.nslabs, 32, 0, st>>>(op, outs, r0, rc, xp, y, ldy, alpha, beta, bz, cjg);
    return cudaGetLastError();
}

// Matrix-free near field ---------------------------------------------------------------------
// The point kernels of H2B_NEAR_LAPLACE / H2B_NEAR_HELMHOLTZ: the entry of (output dof i, input
// dof j) from their squared distance; 0 for coincident points (the self term).
constexpr double kInv4Pi = 0.25 / 3.141592653589793;

template <int KIND, class V> __device__ __forceinline__ V near_entry(double r2, double k);
template <> __device__ __forceinline__ double near_entry<H2B_NEAR_LAPLACE, double>(double r2, double) {
    return r2 > 0.0 ? kInv4Pi * rsqrt(r2) : 0.0;
}
template <> __device__ __forceinline__ cdouble near_entry<H2B_NEAR_LAPLACE, cdouble>(double r2, double) {
    return {r2 > 0.0 ? kInv4Pi * rsqrt(r2) : 0.0, 0.0};
}
template <> __device__ __forceinline__ cdouble near_entry<H2B_NEAR_HELMHOLTZ, cdouble>(double r2, double k) {
    if (!(r2 > 0.0)) return {0.0, 0.0};
    const double r = sqrt(r2);
    double sn, cs;
    sincos(k * r, &sn, &cs);
    const double w = kInv4Pi / r;
    return {cs * w, sn * w};
}

// y[rows(g)] = alpha * op(N_g) x + beta * y[rows(g)] with N's entries computed from the points:
// the block walk of near_rows_kernel (units = (block, 32-column chunk) dealt to the warps), but
// each lane owns rows lane, lane + 32, ... (up to RM per pass, as many as the leaf needs) and
// evaluates its entries column by column; the column's point and x values are broadcast from
// shared memory. N^T has the same entries with the roles of the sides swapped (the kernels are
// symmetric), conj(N^T) for adjoint maps.
template <class V, int KIND, int R, int RM>
__global__ void __launch_bounds__(NEAR_WARPS * 32, 2)
near_free_kernel(NearOp op, DSide outs, DSide ins, const double *__restrict__ pout,
                 const double *__restrict__ pin, double wavenumber, bool cjg, int r0, int rc,
                 const V *__restrict__ x, int64_t ldx, V *__restrict__ y, int64_t ldy, V alpha, V beta,
                 bool beta_zero) {
    constexpr int RPP = 32 * RM;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int g = blockIdx.x;
    const int leaf = op.grp_leaf[g];
    const int o0 = outs.value_ptr[leaf], nr = outs.value_ptr[leaf + 1] - o0;
    const int u0 = op.unit_ptr[g], u1 = op.unit_ptr[g + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    V *xs = reinterpret_cast<V *>(smem_raw) + warp * 32 * R;             // this warp's x chunk
    double *qs = reinterpret_cast<double *>(reinterpret_cast<V *>(smem_raw) + NEAR_WARPS * 32 * R) +
                 warp * 32 * 3;                                             // its column points
    V *part = reinterpret_cast<V *>(reinterpret_cast<double *>(reinterpret_cast<V *>(smem_raw) +
                                                               NEAR_WARPS * 32 * R) + NEAR_WARPS * 32 * 3);
    for (int p0 = 0; p0 < nr; p0 += RPP) {
        const int km = min(RM, (nr - p0 + 31) / 32);  // warp-uniform: row slots in use
        double px[RM], py[RM], pz[RM];
        bool live[RM];
        V acc[RM][R];
#pragma unroll
        for (int k = 0; k < RM; ++k) {
            const int i = p0 + 32 * k + lane;
            live[k] = i < nr;
            const int64_t dof = live[k] ? outs.value[o0 + i] : outs.value[o0];
            px[k] = pout[3 * dof];
            py[k] = pout[3 * dof + 1];
            pz[k] = pout[3 * dof + 2];
#pragma unroll
            for (int q = 0; q < R; ++q) acc[k][q] = V{};
        }
        {
            for (int un = u0 + warp; un < u1; un += NEAR_WARPS) {
                const int jn = op.unit[un].y, c0 = op.unit[un].x;
                __syncwarp();
                {
                    const int64_t dof = lane < jn ? ins.value[c0 + lane] : 0;
#pragma unroll
                    for (int q = 0; q < R; ++q)
                        xs[lane * R + q] = (lane < jn && q < rc) ? x[(int64_t)(r0 + q) * ldx + dof] : V{};
                    qs[3 * lane] = pin[3 * dof];
                    qs[3 * lane + 1] = pin[3 * dof + 1];
                    qs[3 * lane + 2] = pin[3 * dof + 2];
                }
                __syncwarp();
                for (int jj = 0; jj < jn; ++jj) {
                    const double qx = qs[3 * jj], qy = qs[3 * jj + 1], qz = qs[3 * jj + 2];
                    V xv[R];
                    load_x<V, R>(xs + jj * R, xv);
#pragma unroll
                    for (int k = 0; k < RM; ++k) {
                        if (k >= km) break;
                        const double dx = px[k] - qx, dy = py[k] - qy, dz = pz[k] - qz;
                        const V a = near_entry<KIND, V>(fma(dx, dx, fma(dy, dy, dz * dz)), wavenumber);
#pragma unroll
                        for (int q = 0; q < R; ++q) acc[k][q] = fma_c(a, xv[q], acc[k][q], cjg);
                    }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < RM; ++k)
#pragma unroll
            for (int q = 0; q < R; ++q) part[(warp * RPP + 32 * k + lane) * R + q] = acc[k][q];
        __syncthreads();
        const int rows = min(RPP, nr - p0);
        for (int e = threadIdx.x; e < rows * rc; e += blockDim.x) {
            const int i = e / rc, q = e % rc;
            V s = V{};
#pragma unroll
            for (int w = 0; w < NEAR_WARPS; ++w) s = s + part[(w * RPP + i) * R + q];
            V *o = &y[(int64_t)(r0 + q) * ldy + outs.value[o0 + p0 + i]];
            const V v = alpha * s;
            *o = beta_zero ? v : v + beta * *o;
        }
        __syncthreads();
    }
}

// rows per lane and pass: four (128 rows) for one or two right-hand sides, fewer where the
// accumulators of more right-hand sides need the registers
template <class V, int R> struct FreeShape {
    static constexpr bool cplx = sizeof(V) == 16;
    static constexpr int RM = R <= 2 ? 4 : (R <= 8 && !cplx ? 2 : (R <= 4 ? 2 : 1));
};

template <class V, int KIND, int R>
cudaError_t launch_free_t(const NearOp &op, const DSide &outs, const DSide &ins, const double *pout,
                          const double *pin, double k, bool cjg, int r0, int rc, const V *x, int64_t ldx,
                          V *y, int64_t ldy, V alpha, V beta, bool bz, cudaStream_t st) {
    constexpr int RM = FreeShape<V, R>::RM;
    const size_t sm = (size_t)NEAR_WARPS * (32 * R * sizeof(V) + 32 * 3 * sizeof(double) +
                                            (size_t)32 * RM * R * sizeof(V));
    auto kern = near_free_kernel<V, KIND, R, RM>;
    cudaError_t e = cudaSuccess;
    if (sm > 48 * 1024) e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    kern<<<op.ngroups, NEAR_WARPS * 32, sm, st>>>(op, outs, ins, pout, pin, k, cjg, r0, rc, x, ldx, y, ldy,
                                                   alpha, beta, bz);
    return cudaGetLastError();
}

template <class V, int KIND>
cudaError_t near_free_apply_t(const NearOp &op, const DSide &outs, const DSide &ins, const double *pout,
                              const double *pin, double k, bool cjg, int nrhs, const V *x, int64_t ldx,
                              V *y, int64_t ldy, V alpha, V beta, bool bz, cudaStream_t st) {
    if (op.ngroups == 0) return cudaSuccess;
    constexpr int RB = sizeof(V) == 16 ? 8 : 16;  // complex: 16 accumulators would spill
    for (int r0 = 0; r0 < nrhs; r0 += RB) {
        const int rc = std::min(RB, nrhs - r0);
        cudaError_t e;
        if (rc == 1) e = launch_free_t<V, KIND, 1>(op, outs, ins, pout, pin, k, cjg, r0, rc, x, ldx, y, ldy, alpha, beta, bz, st);
        else if (rc == 2) e = launch_free_t<V, KIND, 2>(op, outs, ins, pout, pin, k, cjg, r0, rc, x, ldx, y, ldy, alpha, beta, bz, st);
        else if (rc <= 4) e = launch_free_t<V, KIND, 4>(op, outs, ins, pout, pin, k, cjg, r0, rc, x, ldx, y, ldy, alpha, beta, bz, st);
        else if (rc <= 8) e = launch_free_t<V, KIND, 8>(op, outs, ins, pout, pin, k, cjg, r0, rc, x, ldx, y, ldy, alpha, beta, bz, st);
        else e = launch_free_t<V, KIND, RB>(op, outs, ins, pout, pin, k, cjg, r0, rc, x, ldx, y, ldy, alpha, beta, bz, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Build-time helpers --------------------------------------------------------------------------
// Copy block b (nr x nc, column-major, leading dimension nr) into the padded layout; with
// `transpose`, write its transpose (nc x nr) instead.
template <class V>
__global__ void near_repack_kernel(const V *__restrict__ src, const int64_t *__restrict__ src_off,
                                   const int *__restrict__ blk_row, const int *__restrict__ blk_col,
                                   DSide rows, DSide cols, V *__restrict__ dst,
                                   const int64_t *__restrict__ dst_off, bool transpose) {
    const int b = blockIdx.x;
    const int r = blk_row[b], c = blk_col[b];
    const int nr = rows.value_ptr[r + 1] - rows.value_ptr[r];
    const int nc = cols.value_ptr[c + 1] - cols.value_ptr[c];
    const V *s = src + src_off[b];
    V *d = dst + dst_off[b];
    if (!transpose) {
        const int ld = near_ld(nr, (V *)nullptr);
        for (int64_t e = threadIdx.x; e < (int64_t)ld * nc; e += blockDim.x) {
            const int i = (int)(e % ld), j = (int)(e / ld);
            d[e] = i < nr ? s[i + (int64_t)j * nr] : V{};
        }
    } else {
        const int ld = near_ld(nc, (V *)nullptr);
        for (int64_t e = threadIdx.x; e < (int64_t)ld * nr; e += blockDim.x) {
            const int j = (int)(e % ld), i = (int)(e / ld);
            d[e] = j < nc ? s[i + (int64_t)j * nr] : V{};
        }
    }
}

__device__ __forceinline__ bool same(double a, double b) { return a == b; }
__device__ __forceinline__ bool same(cdouble a, cdouble b) { return a.x == b.x && a.y == b.y; }

// flag stays 1 only if every block equals the transpose of its mirror block
template <class V>
__global__ void near_symcheck_kernel(const V *__restrict__ src, const int64_t *__restrict__ off,
                                     const int *__restrict__ mirror, const int *__restrict__ blk_row,
                                     DSide rows, int *__restrict__ flag) {
    const int b = blockIdx.x;
    const int m = mirror[b];
    const int r = blk_row[b];
    const int nr = rows.value_ptr[r + 1] - rows.value_ptr[r];
    const int nc = rows.value_ptr[blk_row[m] + 1] - rows.value_ptr[blk_row[m]];
    const V *s = src + off[b];
    const V *t = src + off[m];
    bool ok = true;
    for (int64_t e = threadIdx.x; e < (int64_t)nr * nc; e += blockDim.x) {
        const int i = (int)(e % nr), j = (int)(e / nr);
        ok &= same(s[e], t[j + (int64_t)i * nc]);
    }
    if (!__syncthreads_and(ok) && threadIdx.x == 0) *flag = 0;
}

// Pass shape per (field, right-hand sides): MP chunks per pass, UB columns per load batch, MINB
// CTAs per SM for the register budget. Two right-hand sides take two chunks per pass (128 real or
// 64 complex rows); one real right-hand side keeps one chunk and three CTAs per SM (85 registers),
// which streams faster on B200 than the two-chunk pass at two CTAs per SM.
template <class V, int R> struct NearShape {
    static constexpr bool cplx = sizeof(V) == 16;
    static constexpr int MP = R <= 2 ? 2 - (!cplx && R == 1) : 1;
    static constexpr int UB = cplx ? 4 : 8;
    static constexpr int MINB = 2;
};

template <class V, int R>
cudaError_t launch_rows_t(const NearOp &op, const DSide &outs, const DSide &ins, bool cjg, int r0,
                          int rc, const V *x, int64_t ldx, V *y, int64_t ldy, V alpha, V beta,
                          bool bz, cudaStream_t st) {
    constexpr int MP = NearShape<V, R>::MP, UB = NearShape<V, R>::UB, MINB = NearShape<V, R>::MINB;
    constexpr int RPP = 32 * NearVec<V>::RPL * MP;
    const size_t sm = (size_t)NEAR_WARPS * (32 + RPP) * R * sizeof(V);
    auto kern = near_rows_kernel<V, R, MP, UB, MINB>;
    cudaError_t e = cudaSuccess;
    if (sm > 48 * 1024) e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    kern<<<op.ngroups, NEAR_WARPS * 32, sm, st>>>(op, outs, ins, cjg, r0, rc, x, ldx, y, ldy, alpha, beta, bz);
    return cudaGetLastError();
}

template <class V>
cudaError_t near_apply_t(const NearOp &op, const DSide &outs, const DSide &ins, bool cjg, int nrhs,
                         const V *x, int64_t ldx, V *y, int64_t ldy, V alpha, V beta, bool bz,
                         double *xp, cudaStream_t st) {
    if (op.ngroups == 0) return cudaSuccess;
    if constexpr (std::is_same<V, cdouble>::value) {
        // complex blocks, 8 or more right-hand sides (workspaces that size carry the gather
        // buffer): FP64 tensor cores, 16 right-hand sides per pass over the blocks (32 would hold
        // 64 FP64 accumulators per lane and spill)
        const int rb = near_rhs_block(nrhs);
        int r0 = 0;
        for (; xp && r0 < nrhs && nrhs - r0 >= 8; r0 += rb) {
            const int rc = std::min(rb, nrhs - r0);
            cudaError_t e = launch_slab_mma_c<16>(op, outs, ins, cjg, r0, rc, x, ldx, (cdouble *)xp, y, ldy, alpha,
                                                  beta, bz, st);
            if (e != cudaSuccess) return e;
        }
        x += r0 * ldx;
        y += r0 * ldy;
        nrhs -= r0;
    }
    for (int r0 = 0; r0 < nrhs; r0 += 16) {
        const int rc = std::min(16, nrhs - r0);
        cudaError_t e;
        if constexpr (std::is_same<V, double>::value) {
            // real blocks, 8 or more right-hand sides: FP64 tensor-core MMA
            // 8 or more right-hand sides (workspaces that size carry the gather buffer): tensor cores
            if (rc > 8 && xp) {
                e = launch_rows_mma<2>(op, outs, ins, r0, rc, x, ldx, xp, y, ldy, alpha, beta, bz, st);
                if (e != cudaSuccess) return e;
                continue;
            }
            if (rc == 8 && xp) {
                e = launch_rows_mma<1>(op, outs, ins, r0, rc, x, ldx, xp, y, ldy, alpha, beta, bz, st);
                if (e != cudaSuccess) return e;
                continue;
            }
        }
        if (rc == 1) e = launch_rows_t<V, 1>(op, outs, ins, cjg, r0, rc, x, ldx, y, ldy, alpha, beta, bz, st);
        else if (rc == 2) e = launch_rows_t<V, 2>(op, outs, ins, cjg, r0, rc, x, ldx, y, ldy, alpha, beta, bz, st);
        else if (rc <= 4) e = launch_rows_t<V, 4>(op, outs, ins, cjg, r0, rc, x, ldx, y, ldy, alpha, beta, bz, st);
        else if (rc <= 8) e = launch_rows_t<V, 8>(op, outs, ins, cjg, r0, rc, x, ldx, y, ldy, alpha, beta, bz, st);
        else e = launch_rows_t<V, 16>(op, outs, ins, cjg, r0, rc, x, ldx, y, ldy, alpha, beta, bz, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

int64_t near_padded_ld(bool cplx, int n) { return cplx ? n : n + (n & 1); }

int near_rhs_block(int) { return 16; }

cudaError_t launch_near_repack(bool cplx, const void *src, const int64_t *src_off, const int *blk_row,
                               const int *blk_col, const DSide &rows, const DSide &cols, void *dst,
                               const int64_t *dst_off, int nblocks, bool transpose, cudaStream_t st) {
    if (nblocks == 0) return cudaSuccess;
    if (cplx)
        near_repack_kernel<cdouble><<<nblocks, 256, 0, st>>>(static_cast<const cdouble *>(src), src_off, blk_row,
                                                             blk_col, rows, cols, static_cast<cdouble *>(dst),
                                                             dst_off, transpose);
    else
        near_repack_kernel<double><<<nblocks, 256, 0, st>>>(static_cast<const double *>(src), src_off, blk_row,
                                                            blk_col, rows, cols, static_cast<double *>(dst),
                                                            dst_off, transpose);
    return cudaGetLastError();
}

cudaError_t launch_near_symcheck(bool cplx, const void *src, const int64_t *off, const int *mirror,
                                 const int *blk_row, const DSide &rows, int nblocks, int *flag,
                                 cudaStream_t st) {
    if (nblocks == 0) return cudaSuccess;
    if (cplx)
        near_symcheck_kernel<cdouble><<<nblocks, 256, 0, st>>>(static_cast<const cdouble *>(src), off, mirror,
                                                               blk_row, rows, flag);
    else
        near_symcheck_kernel<double><<<nblocks, 256, 0, st>>>(static_cast<const double *>(src), off, mirror,
                                                              blk_row, rows, flag);
    return cudaGetLastError();
}

cudaError_t launch_near(bool cplx, int mode, const DNear &n, const DSide &test, const DSide &trial,
                        int nrhs, const void *x, int64_t ldx, void *y, int64_t ldy, cdouble alpha,
                        cdouble beta, void *xp, cudaStream_t st) {
    const bool fwd_op = mode == H2B_FORWARD || n.symmetric;
    const NearOp &op = fwd_op ? n.fwd : n.tr;
    const DSide &outs = fwd_op ? test : trial;
    const DSide &ins = fwd_op ? trial : test;
    const bool cjg = mode == H2B_ADJOINT && cplx;
    if (n.kind != H2B_NEAR_STORED) {
        const double *pout = fwd_op ? n.test_pts : n.trial_pts;
        const double *pin = fwd_op ? n.trial_pts : n.test_pts;
        const bool bz = beta.x == 0.0 && beta.y == 0.0;
        const cdouble *xc = static_cast<const cdouble *>(x);
        cdouble *yc = static_cast<cdouble *>(y);
        if (n.kind == H2B_NEAR_HELMHOLTZ)
            return near_free_apply_t<cdouble, H2B_NEAR_HELMHOLTZ>(op, outs, ins, pout, pin, n.wavenumber, cjg,
                                                                   nrhs, xc, ldx, yc, ldy, alpha, beta, bz, st);
        if (cplx)
            return near_free_apply_t<cdouble, H2B_NEAR_LAPLACE>(op, outs, ins, pout, pin, 0.0, cjg, nrhs, xc,
                                                                 ldx, yc, ldy, alpha, beta, bz, st);
        return near_free_apply_t<double, H2B_NEAR_LAPLACE>(op, outs, ins, pout, pin, 0.0, false, nrhs,
                                                            static_cast<const double *>(x), ldx,
                                                            static_cast<double *>(y), ldy, alpha.x, beta.x,
                                                            beta.x == 0.0, st);
    }
    if (cplx)
        return near_apply_t<cdouble>(op, outs, ins, cjg, nrhs, static_cast<const cdouble *>(x), ldx,
                                     static_cast<cdouble *>(y), ldy, alpha, beta,
                                     beta.x == 0.0 && beta.y == 0.0, static_cast<double *>(xp), st);
    return near_apply_t<double>(op, outs, ins, false, nrhs, static_cast<const double *>(x), ldx,
                                static_cast<double *>(y), ldy, alpha.x, beta.x, beta.x == 0.0,
                                static_cast<double *>(xp), st);
}

}  // namespace h2b
