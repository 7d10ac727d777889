// Kernels of the H2 matrix-vector product on sm_100a.
//
// One launch per traversal phase (and per level where the phase depends on the level above or
// below), each over a flat node list built from the plans when the core is created:
//   leaf_aggregate     A1  aggregateleaf!      src/farinteractions/traversalhelpers.jl:36-42
//   transfer_up        A2  i2ipass!            traversalhelpers.jl:49-75
//   toeplitz_in        A3  modulate_in!        src/moments/toeplitz/toeplitzmul.jl:290-297
//   i2o                B1/B2 translateintonode! traversalhelpers.jl:167-219
//   toeplitz_out       B3  modulate_out!       toeplitzmul.jl:299-315
//   transfer_down      C1  O2O                 src/farinteractions/disaggregation.jl:244-271
//   leaf_disaggregate  C2  disaggregateleaf!   traversalhelpers.jl:84-96
//   (near field: h2b_near.cu)
// Column-major operands are read along their contiguous dimension by consecutive threads
// (thread per row for A x), or by the lanes of one warp with a shuffle reduction (warp per
// output for A^T x), so every global read is coalesced.

#include <algorithm>
#include <type_traits>

#include "h2b_internal.cuh"

namespace h2b {

namespace {


__device__ __forceinline__ int ncoef_of(const DSide &s, int lvl) {
    return s.shape[3 * lvl] * s.shape[3 * lvl + 1] * s.shape[3 * lvl + 2];
}

// Bound on every intermediate of a separable contraction between levels lp and lp + 1.
__device__ __forceinline__ int sep_bound(const DSide &s, int lp) {
    int b = 1;
    for (int d = 0; d < 3; ++d) b *= max(s.shape[3 * lp + d], s.shape[3 * (lp + 1) + d]);
    return b;
}

// ---------------------------------------------------------------------------------------------
// Per-node small products on all right-hand sides at once: acc (+)= op(M) X over a tile of at most
// TG_M output rows and TG_Q right-hand sides. op(M)[i, k] = M[i + k*ldm] (trans = false) or
// M[k + i*ldm] (trans = true), conjugated when cjg. M and X are staged through shared memory in
// chunks of TG_K along k, loaded along their contiguous dimension, in the FP64 accumulation type.
// Thread t owns outputs o = t + j*blockDim.x, (i, q) = (o % mt, o / mt).
// ---------------------------------------------------------------------------------------------
constexpr int TG_M = 64, TG_K = 32, TG_Q = 16, TG_LD = TG_K + 1;
constexpr int TG_O = TG_M * TG_Q / 256;  // outputs per thread at 256 threads

// General form: mload(i, k) returns op(M)[i, k] in A; `kfast` says consecutive k are contiguous in
// memory (so staging walks k fastest), otherwise consecutive i are.
template <class A, class MLoad, class XLoad>
__device__ __forceinline__ void tile_gemm_l(bool kfast, int m0, int mt, int kk, int nq, MLoad mload,
                                            XLoad xload, A *Ms, A *Xs, A (&acc)[TG_O]) {
    for (int k0 = 0; k0 < kk; k0 += TG_K) {
        const int kc = min(TG_K, kk - k0);
        __syncthreads();
        if (kfast) {
            for (int idx = threadIdx.x; idx < mt * TG_K; idx += blockDim.x) {
                const int k = idx % TG_K, i = idx / TG_K;
                Ms[i * TG_LD + k] = k < kc ? mload(m0 + i, k0 + k) : A{};
            }
        } else {
            for (int idx = threadIdx.x; idx < mt * TG_K; idx += blockDim.x) {
                const int i = idx % mt, k = idx / mt;
                Ms[i * TG_LD + k] = k < kc ? mload(m0 + i, k0 + k) : A{};
            }
        }
        for (int idx = threadIdx.x; idx < TG_K * nq; idx += blockDim.x) {
            const int k = idx % TG_K, q = idx / TG_K;
            Xs[k * TG_Q + q] = k < kc ? xload(k0 + k, q) : A{};
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < TG_O; ++j) {
            const int o = threadIdx.x + j * blockDim.x;
            if (o < mt * nq) {
                const int i = o % mt, q = o / mt;
                A sacc = acc[j];
#pragma unroll 8
                for (int k = 0; k < TG_K; ++k) sacc = sacc + Ms[i * TG_LD + k] * Xs[k * TG_Q + q];
                acc[j] = sacc;
            }
        }
    }
}

// The same tile product on the FP64 tensor cores (mma.sync m8n8k4 .f64): warp w owns output rows
// 8w..8w+7 of the tile (TG_M = 64 rows for 8 warps) and both 8-wide right-hand-side halves of
// TG_Q. Complex tiles take four real products per k-step (re = ar br - ai bi, im = ar bi + ai br).
// Fragment layout (PTX ISA, m8n8k4 .f64): A[lane/4][lane%4], B[lane%4][lane/4],
// C[lane/4][2*(lane%4) + i]. Rows past mt and columns past nq compute on stale shared memory and
// are never stored; k past the chunk is zero-filled, as in tile_gemm_l.
__device__ __forceinline__ void dmma8(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

template <class A> struct MmaAcc;
template <> struct MmaAcc<double> {
    double c[2][2];
    __device__ void zero() { c[0][0] = c[0][1] = c[1][0] = c[1][1] = 0.0; }
    __device__ void step(double a, const double (&b)[2]) {
#pragma unroll
        for (int u = 0; u < 2; ++u) dmma8(c[u], a, b[u]);
    }
    __device__ double get(int u, int h) const { return c[u][h]; }
};
template <> struct MmaAcc<cdouble> {
    double re[2][2], im[2][2];
    __device__ void zero() {
#pragma unroll
        for (int u = 0; u < 2; ++u) re[u][0] = re[u][1] = im[u][0] = im[u][1] = 0.0;
    }
    __device__ void step(cdouble a, const cdouble (&b)[2]) {
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            dmma8(re[u], a.x, b[u].x);
            dmma8(re[u], -a.y, b[u].y);
            dmma8(im[u], a.x, b[u].y);
            dmma8(im[u], a.y, b[u].x);
        }
    }
    __device__ cdouble get(int u, int h) const { return {re[u][h], im[u][h]}; }
};

template <class A, class MLoad, class XLoad>
__device__ __forceinline__ void tile_gemm_mma_l(bool kfast, int m0, int mt, int kk, int nq, MLoad mload,
                                                XLoad xload, A *Ms, A *Xs, MmaAcc<A> &acc) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g4 = lane >> 2, t4 = lane & 3;
    for (int k0 = 0; k0 < kk; k0 += TG_K) {
        const int kc = min(TG_K, kk - k0);
        __syncthreads();
        if (kfast) {
            for (int idx = threadIdx.x; idx < mt * TG_K; idx += blockDim.x) {
                const int k = idx % TG_K, i = idx / TG_K;
                Ms[i * TG_LD + k] = k < kc ? mload(m0 + i, k0 + k) : A{};
            }
        } else {
            for (int idx = threadIdx.x; idx < mt * TG_K; idx += blockDim.x) {
                const int i = idx % mt, k = idx / mt;
                Ms[i * TG_LD + k] = k < kc ? mload(m0 + i, k0 + k) : A{};
            }
        }
        for (int idx = threadIdx.x; idx < TG_K * nq; idx += blockDim.x) {
            const int k = idx % TG_K, q = idx / TG_K;
            Xs[k * TG_Q + q] = k < kc ? xload(k0 + k, q) : A{};
        }
        __syncthreads();
        if (8 * warp < mt) {
            const A *mrow = Ms + (8 * warp + g4) * TG_LD + t4;
            const A *xcol = Xs + t4 * TG_Q + g4;
#pragma unroll
            for (int k = 0; k < TG_K; k += 4) {
                const A a = mrow[k];
                const A b[2] = {xcol[k * TG_Q], xcol[k * TG_Q + 8]};
                acc.step(a, b);
            }
        }
    }
}

// f(i, q, value) for every element of the warp's C fragments inside the mt x nq tile
template <class A, class F>
__device__ __forceinline__ void mma_store(const MmaAcc<A> &acc, int mt, int nq, F f) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int i = 8 * warp + (lane >> 2);
    if (i >= mt) return;
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int q = 8 * u + 2 * (lane & 3) + h;
            if (q < nq) f(i, q, acc.get(u, h));
        }
}

// A 64 x 16 output tile on the FP64 tensor cores held by ONE warp, operands read straight from
// global memory (no shared-memory staging, no block barrier): acc += op(A) B, 8 row tiles x 2
// column tiles of mma.sync m8n8k4 per k step of 4. a(i, k) and b(k, q) return the operands; rows
// >= M, columns >= nq and k >= K read as zero. Lane fragments as in dmma8: A[g4][t4], B[t4][g4],
// so acc[t][u][h] is C[8t + g4][8u + 2 t4 + h]. Each k step issues its 10 loads per lane before
// its 16 products, and the loop is unrolled twice, so loads of the next step overlap the products.
// For the small real products of the transfers and leaves with 2-16 right-hand sides, where a
// CTA-wide staged tile waits on one load round trip per 32-wide chunk.
template <class ALoad, class BLoad>
__device__ __forceinline__ void warp_mma64x16(int M, int K, int nq, ALoad a, BLoad b, double (&acc)[8][2][2]) {
    const int lane = threadIdx.x & 31, g4 = lane >> 2, t4 = lane & 3;
#pragma unroll 2
    for (int k0 = 0; k0 < K; k0 += 4) {
        const int k = k0 + t4;
        const bool kin = k < K;
        double af[8], bf[2];
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const int i = 8 * t + g4;
            af[t] = kin && i < M ? a(i, k) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int q = 8 * u + g4;
            bf[u] = kin && q < nq ? b(k, q) : 0.0;
        }
#pragma unroll
        for (int t = 0; t < 8; ++t)
#pragma unroll
            for (int u = 0; u < 2; ++u) dmma8(acc[t][u], af[t], bf[u]);
    }
}

__device__ __forceinline__ void warp_acc_zero(double (&acc)[8][2][2]) {
#pragma unroll
    for (int t = 0; t < 8; ++t)
#pragma unroll
        for (int u = 0; u < 2; ++u) acc[t][u][0] = acc[t][u][1] = 0.0;
}

// f(i, q, value) for every element of the warp's tile inside M x nq
template <class F>
__device__ __forceinline__ void warp_acc_store(const double (&acc)[8][2][2], int M, int nq, F f) {
    const int lane = threadIdx.x & 31, g4 = lane >> 2, t4 = lane & 3;
#pragma unroll
    for (int t = 0; t < 8; ++t)
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int i = 8 * t + g4, q = 8 * u + 2 * t4 + h;
                if (i < M && q < nq) f(i, q, acc[t][u][h]);
            }
}

// op(M)[i, k] = M[i + k*ldm] (trans = false) or M[k + i*ldm] (trans = true), conjugated when cjg.
template <class T, class A, class XLoad>
__device__ __forceinline__ void tile_gemm(const T *__restrict__ M, int64_t ldm, bool trans, bool cjg, int m0,
                                          int mt, int kk, int nq, XLoad xload, A *Ms, A *Xs, A (&acc)[TG_O]) {
    if (trans)
        tile_gemm_l(true, m0, mt, kk, nq, [&](int i, int k) -> A { return wide(cj(M[k + (int64_t)i * ldm], cjg)); },
                    xload, Ms, Xs, acc);
    else
        tile_gemm_l(false, m0, mt, kk, nq, [&](int i, int k) -> A { return wide(cj(M[i + (int64_t)k * ldm], cjg)); },
                    xload, Ms, Xs, acc);
}

template <class A>
__device__ __forceinline__ void tile_zero(A (&acc)[TG_O]) {
#pragma unroll
    for (int j = 0; j < TG_O; ++j) acc[j] = A{};
}

// smem for tile_gemm and tile_gemm_mma_l: Ms [TG_M][TG_LD] + Xs [TG_K][TG_Q]
template <class A>
constexpr size_t tile_smem() { return (size_t)(TG_M * TG_LD + TG_K * TG_Q) * sizeof(A); }

// ---------------------------------------------------------------------------------------------
// A1: m_leaf[c][r] = op(C_c) x[values]   (op = conj for adjoint maps with conjugating leaves);
// RCH right-hand sides share each pass over the collection
// ---------------------------------------------------------------------------------------------
template <class T, class V, bool MMA>
__global__ void __launch_bounds__(256)
leaf_aggregate_kernel(DMap m, DSide s, const int *__restrict__ leaves, bool conjc, int nrhs,
                      const V *__restrict__ x, int64_t ldx, T *__restrict__ am) {
    using A = typename ScalarTraits<T>::Acc;  // == V
    extern __shared__ unsigned char smem_raw[];
    A *Ms = reinterpret_cast<A *>(smem_raw), *Xs = Ms + TG_M * TG_LD;
    const int leaf = leaves[blockIdx.x];
    const int nc = ncoef_of(s, s.level[leaf]);
    const int v0 = s.value_ptr[leaf], nv = s.value_ptr[leaf + 1] - v0;
    const T *C = static_cast<const T *>(s.coll) + s.coll_off[leaf];
    T *mom = am + s.mom_off[leaf] * nrhs;
    for (int c = 0; c < m.ncomp; ++c)
        for (int q0 = 0; q0 < nrhs; q0 += TG_Q) {
            const int nq = min(TG_Q, nrhs - q0);
            for (int m0 = 0; m0 < nc; m0 += TG_M) {
                const int mt = min(TG_M, nc - m0);
                const T *Cc = C + (int64_t)c * nc * nv;
                if constexpr (!MMA) {  // one right-hand side: FMA tile (an MMA would idle 7 of 8 columns)
                    A acc[TG_O];
                    tile_zero(acc);
                    tile_gemm(Cc, nc, false, conjc, m0, mt, nv, nq,
                              [&](int k, int q) -> A { return x[(int64_t)(q0 + q) * ldx + s.value[v0 + k]]; },
                              Ms, Xs, acc);
#pragma unroll
                    for (int j = 0; j < TG_O; ++j) {
                        const int o = threadIdx.x + j * blockDim.x;
                        if (o < mt * nq)
                            narrow(acc[j], mom[((int64_t)c * nrhs + q0 + o / mt) * nc + m0 + o % mt]);
                    }
                } else {
                MmaAcc<A> acc;  // FP64 tensor cores (256 threads: 8 warps x 8 rows)
                acc.zero();
                tile_gemm_mma_l(false, m0, mt, nv, nq,
                                [&](int i, int k) -> A { return wide(cj(Cc[i + (int64_t)k * nc], conjc)); },
                                [&](int k, int q) -> A { return x[(int64_t)(q0 + q) * ldx + s.value[v0 + k]]; },
                                Ms, Xs, acc);
                mma_store(acc, mt, nq, [&](int i, int q, A v) {
                    narrow(v, mom[((int64_t)c * nrhs + q0 + q) * nc + m0 + i]);
                });
                }
            }
        }
}

// ---------------------------------------------------------------------------------------------
// Separable contraction of one moment component in shared memory: out (+)= op(M_dim..M_1) in,
// axes from `dim` down to 1 (src/maps/leveltranslator.jl:200-265). op: transposed factors when
// `tr`, conjugated when `cjg`. Factor ax is stored sp[ax] x sc[ax] (parent x child), column-major.
// Buffers a, b hold max(prod(fin), prod(fout)) elements; in is consumed from `a`.
// ---------------------------------------------------------------------------------------------
template <class T, class A, class O>
__device__ void separable_block(const T *M, const int *sp, const int *sc, int dim, bool up, bool cjg,
                                A *a, A *b, O *out, bool accumulate) {
    int cur[3], fin[3], fout[3];
    for (int d = 0; d < 3; ++d) {
        fin[d] = up ? sc[d] : sp[d];
        fout[d] = up ? sp[d] : sc[d];
        cur[d] = fin[d];
    }
    const T *fac[3];
    int64_t o = 0;
    for (int d = 0; d < dim; ++d) {
        fac[d] = M + o;
        o += (int64_t)sp[d] * sc[d];
    }
    for (int ax = dim - 1; ax >= 0; --ax) {
        int nxt[3] = {cur[0], cur[1], cur[2]};
        nxt[ax] = fout[ax];
        const int total = nxt[0] * nxt[1] * nxt[2];
        const int ld = sp[ax];
        for (int e = threadIdx.x; e < total; e += blockDim.x) {
            int idx[3] = {e % nxt[0], (e / nxt[0]) % nxt[1], e / (nxt[0] * nxt[1])};
            const int row = idx[ax];
            A acc = sc_zero<A>();
            for (int k = 0; k < cur[ax]; ++k) {
                int src[3] = {idx[0], idx[1], idx[2]};
                src[ax] = k;
                // up: op(M)[row,k] = M[row + k*ld]; down: M^T[row,k] = M[k + row*ld]
                const T mk = up ? fac[ax][row + k * ld] : fac[ax][k + row * ld];
                acc = acc + wide(cj(mk, cjg)) * a[src[0] + cur[0] * (src[1] + cur[1] * src[2])];
            }
            b[e] = acc;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < total; e += blockDim.x) a[e] = b[e];
        __syncthreads();
        cur[0] = nxt[0]; cur[1] = nxt[1]; cur[2] = nxt[2];
    }
    const int total = fout[0] * fout[1] * fout[2];
    for (int e = threadIdx.x; e < total; e += blockDim.x) narrow(accumulate ? wide(out[e]) + a[e] : a[e], out[e]);
    __syncthreads();
}

// ---------------------------------------------------------------------------------------------
// Separable level transfers (SeparableI2I, src/maps/leveltranslator.jl:168-265) on blocks of
// right-hand sides: one CTA per parent (upward: m_p = sum over children of op(T_c) m_c, first child
// overwriting) or per child (downward: l_c (+)= op(T_c)^T l_p, accumulating where the child already
// received I2O contributions). A chunk of `qc` moment columns is contracted axis by axis in
// shared memory (axes dim .. 1, one barrier per axis, ping-pong buffers); each thread computes
// whole output elements of the axis pass, so the work of one barrier is qc times that of one column.
// ---------------------------------------------------------------------------------------------
template <class T, bool UP>
__global__ void __launch_bounds__(256)
transfer_sep_kernel(DMap m, DSide s, const int *__restrict__ nodes, const uint8_t *__restrict__ received,
                    bool conjt, int nrhs, T *__restrict__ mom, int qc_max, int bufsz) {
    using A = typename ScalarTraits<T>::Acc;
    extern __shared__ unsigned char smem_raw[];
    A *X = reinterpret_cast<A *>(smem_raw), *Y = X + (size_t)qc_max * bufsz, *Acc = Y + (size_t)qc_max * bufsz;
    const int node = nodes[blockIdx.x];
    const int lp = UP ? s.level[node] : s.level[node] - 1, lc = lp + 1;
    const int *sp = &s.shape[3 * lp], *sc = &s.shape[3 * lc];
    int fin[3], fout[3];
    for (int d = 0; d < 3; ++d) {
        fin[d] = UP ? sc[d] : sp[d];
        fout[d] = UP ? sp[d] : sc[d];
    }
    const int nin = fin[0] * fin[1] * fin[2], nout = fout[0] * fout[1] * fout[2];
    const int nq = m.ncomp * nrhs;
    const int c0 = UP ? s.child_ptr[node] : 0, c1 = UP ? s.child_ptr[node + 1] : 1;
    T *dst = mom + s.mom_off[node] * nrhs;
    const bool acc_dst = !UP && received[node] != 0;
    for (int q0 = 0; q0 < nq; q0 += qc_max) {
        const int qc = min(qc_max, nq - q0);
        A *res = X;
        for (int k = c0; k < c1; ++k) {
            const int ch = UP ? s.child[k] : node;  // the transfer belongs to the child
            const T *src = UP ? mom + s.mom_off[ch] * nrhs : mom + s.mom_off[s.parent[node]] * nrhs;
            const T *M = static_cast<const T *>(s.tr) + s.tr_off[lc * m.nsectors + s.sector[ch]];
            const T *fac[3];
            int64_t o = 0;
            for (int d = 0; d < m.dim; ++d) {
                fac[d] = M + o;
                o += (int64_t)sp[d] * sc[d];
            }
            for (int e = threadIdx.x; e < qc * nin; e += blockDim.x) {
                const int q = e / nin, i = e - q * nin;
                X[q * bufsz + i] = wide(src[(int64_t)(q0 + q) * nin + i]);
            }
            __syncthreads();
            int cur[3] = {fin[0], fin[1], fin[2]};
            A *a = X, *b = Y;
            for (int ax = m.dim - 1; ax >= 0; --ax) {
                int nxt[3] = {cur[0], cur[1], cur[2]};
                nxt[ax] = fout[ax];
                const int tot = nxt[0] * nxt[1] * nxt[2], ld = sp[ax], kk = cur[ax];
                const int sstr = ax == 0 ? 1 : (ax == 1 ? cur[0] : cur[0] * cur[1]);  // input stride along ax
                for (int e = threadIdx.x; e < qc * tot; e += blockDim.x) {
                    const int q = e / tot, f = e - q * tot;
                    const int i0 = f % nxt[0], i1 = (f / nxt[0]) % nxt[1], i2 = f / (nxt[0] * nxt[1]);
                    const int row = ax == 0 ? i0 : (ax == 1 ? i1 : i2);
                    int base = i0 + cur[0] * (i1 + cur[1] * i2);  // the input index with i[ax] = 0
                    base -= row * sstr;
                    const A *in = a + q * bufsz + base;
                    A acc = sc_zero<A>();
                    for (int j = 0; j < kk; ++j) {
                        // up: op(M)[row, j] = M[row + j ld]; down: M^T[row, j] = M[j + row ld]
                        const T mk = UP ? fac[ax][row + j * ld] : fac[ax][j + row * ld];
                        acc = acc + wide(cj(mk, conjt)) * in[j * sstr];
                    }
                    b[q * bufsz + f] = acc;
                }
                __syncthreads();
                A *t = a;
                a = b;
                b = t;
                cur[0] = nxt[0];
                cur[1] = nxt[1];
                cur[2] = nxt[2];
            }
            res = a;
            if (UP && c1 - c0 > 1) {
                for (int e = threadIdx.x; e < qc * nout; e += blockDim.x) {
                    const int q = e / nout, i = e - q * nout;
                    Acc[q * bufsz + i] = (k == c0 ? sc_zero<A>() : Acc[q * bufsz + i]) + a[q * bufsz + i];
                }
                res = Acc;
                __syncthreads();
            }
        }
        for (int e = threadIdx.x; e < qc * nout; e += blockDim.x) {
            const int q = e / nout, i = e - q * nout;
            T *o = dst + (int64_t)(q0 + q) * nout + i;
            narrow(acc_dst ? wide(*o) + res[q * bufsz + i] : res[q * bufsz + i], *o);
        }
        __syncthreads();
    }
}

template <class T, bool UP>
cudaError_t launch_transfer_sep(const DMap &m, const DSide &s, const int *nodes, int nnodes, const uint8_t *received,
                                bool conjt, int nrhs, void *mom, int maxsep, cudaStream_t st) {
    using A = typename ScalarTraits<T>::Acc;
    const int nq = m.ncomp * nrhs;
    // moment columns per chunk: three buffers of maxsep accumulators each within 48 KB
    const int qc = std::max(1, std::min(nq, (int)((48 * 1024) / (3 * (size_t)maxsep * sizeof(A)))));
    const size_t sm = 3 * (size_t)qc * maxsep * sizeof(A);
    transfer_sep_kernel<T, UP><<<nnodes, 256, sm, st>>>(m, s, nodes, received, conjt, nrhs, static_cast<T *>(mom),
                                                        qc, maxsep);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// A2: m_p = sum over children of op(T_{level(c), sector(c)}) m_c, first child overwriting.
// ---------------------------------------------------------------------------------------------
template <class T, bool MMA>
__global__ void transfer_up_kernel(DMap m, DSide s, const int *__restrict__ nodes, bool conjt,
                                   int nrhs, T *__restrict__ am) {
    using A = typename ScalarTraits<T>::Acc;
    extern __shared__ unsigned char smem_raw[];
    A *sm = reinterpret_cast<A *>(smem_raw);
    const int p = nodes[blockIdx.x];
    const int lp = s.level[p], lc = lp + 1;
    const int nout = ncoef_of(s, lp), nin = ncoef_of(s, lc);
    T *mp = am + s.mom_off[p] * nrhs;
    const int c0 = s.child_ptr[p], c1 = s.child_ptr[p + 1];
    const int nq = m.ncomp * nrhs;
    if (m.transfer_kind == H2B_TRANSFER_DENSE && nq == 1) {
        // one right-hand side: children split over `ns` thread groups of `npad` threads reading
        // their transfers directly (coalesced over the output row), partial sums reduced in smem
        const int npad = ((nout + 31) / 32) * 32;
        const int ns = npad <= (int)blockDim.x ? (int)blockDim.x / npad : 1;
        const int sidx = threadIdx.x / npad;
        for (int a0 = 0; a0 < nout; a0 += (ns > 1 ? npad : (int)blockDim.x)) {
            const int a = a0 + (ns > 1 ? (int)threadIdx.x % npad : (int)threadIdx.x);
            A acc = sc_zero<A>();
            if (sidx < ns && a < nout)
                for (int k = c0 + sidx; k < c1; k += ns) {
                    const int ch = s.child[k];
                    const T *Tk = static_cast<const T *>(s.tr) + s.tr_off[lc * m.nsectors + s.sector[ch]];
                    const T *mc = am + s.mom_off[ch] * nrhs;
#pragma unroll 4
                    for (int b = 0; b < nin; ++b) acc = acc + wide(cj(Tk[a + (int64_t)b * nout], conjt)) * wide(mc[b]);
                }
            if (ns > 1) {
                if (sidx < ns) sm[sidx * npad + (threadIdx.x % npad)] = acc;
                __syncthreads();
                if (threadIdx.x < npad && a0 + threadIdx.x < nout) {
                    A sum = sm[threadIdx.x];
                    for (int w = 1; w < ns; ++w) sum = sum + sm[w * npad + threadIdx.x];
                    narrow(sum, mp[a0 + threadIdx.x]);
                }
                __syncthreads();
            } else if (a < nout) {
                narrow(acc, mp[a]);
            }
        }
        return;
    }
    if (m.transfer_kind == H2B_TRANSFER_DENSE) {
        A *Ms = sm, *Xs = sm + TG_M * TG_LD;
        for (int q0 = 0; q0 < nq; q0 += TG_Q) {
            const int nqc = min(TG_Q, nq - q0);
            for (int m0 = 0; m0 < nout; m0 += TG_M) {
                const int mt = min(TG_M, nout - m0);
                if constexpr (MMA) {
                    MmaAcc<A> acc;  // FP64 tensor cores (256 threads: 8 warps x 8 rows)
                    acc.zero();
                    for (int k = c0; k < c1; ++k) {
                        const int ch = s.child[k];
                        const T *Tk = static_cast<const T *>(s.tr) + s.tr_off[lc * m.nsectors + s.sector[ch]];
                        const T *mc = am + s.mom_off[ch] * nrhs;
                        tile_gemm_mma_l(false, m0, mt, nin, nqc,
                                        [&](int i, int kk) -> A { return wide(cj(Tk[i + (int64_t)kk * nout], conjt)); },
                                        [&](int kk, int q) -> A { return wide(mc[(int64_t)(q0 + q) * nin + kk]); },
                                        Ms, Xs, acc);
                    }
                    mma_store(acc, mt, nqc, [&](int i, int q, A v) { narrow(v, mp[(int64_t)(q0 + q) * nout + m0 + i]); });
                } else {
                    A acc[TG_O];
                    tile_zero(acc);
                    for (int k = c0; k < c1; ++k) {
                        const int ch = s.child[k];
                        const T *Tk = static_cast<const T *>(s.tr) + s.tr_off[lc * m.nsectors + s.sector[ch]];
                        const T *mc = am + s.mom_off[ch] * nrhs;
                        tile_gemm(Tk, nout, false, conjt, m0, mt, nin, nqc,
                                  [&](int kk, int q) -> A { return wide(mc[(int64_t)(q0 + q) * nin + kk]); }, Ms, Xs,
                                  acc);
                    }
#pragma unroll
                    for (int j = 0; j < TG_O; ++j) {
                        const int o = threadIdx.x + j * blockDim.x;
                        if (o < mt * nqc) narrow(acc[j], mp[(int64_t)(q0 + o / mt) * nout + m0 + o % mt]);
                    }
                }
            }
        }
        return;
    }
    const int mx = sep_bound(s, lp);
    A *bufa = sm, *bufb = sm + mx, *acc = sm + 2 * mx;
    for (int q = 0; q < nq; ++q) {
        for (int k = c0; k < c1; ++k) {
            const int ch = s.child[k];
            const T *Tk = static_cast<const T *>(s.tr) + s.tr_off[lc * m.nsectors + s.sector[ch]];
            const T *mc = am + s.mom_off[ch] * nrhs + (int64_t)q * nin;
            for (int e = threadIdx.x; e < nin; e += blockDim.x) bufa[e] = wide(mc[e]);
            __syncthreads();
            separable_block(Tk, &s.shape[3 * lp], &s.shape[3 * lc], m.dim, true, conjt, bufa, bufb,
                            acc, k != c0);
        }
        for (int e = threadIdx.x; e < nout; e += blockDim.x) narrow(acc[e], mp[(int64_t)q * nout + e]);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Real maps, dense transfers and leaf collections of at most 64 coefficients, 2-16 right-hand
// sides: the same products one warp per child / leaf (warp_mma64x16). A2 sums a parent's children
// in a fixed order (warp w holds child w) through shared memory; C1 and A1 write their tiles from
// registers.
// ---------------------------------------------------------------------------------------------
constexpr int WARP_TILE = 64 * 16;  // doubles of one warp's 64 x 16 tile

template <class T>
__global__ void __launch_bounds__(256)
transfer_up_warp_kernel(DMap m, DSide s, const int *__restrict__ nodes, int nrhs, T *__restrict__ am) {
    extern __shared__ double wpart[];  // [8 warps][q * 64 + i]
    const int p = nodes[blockIdx.x];
    const int lp = s.level[p], lc = lp + 1;
    const int nout = ncoef_of(s, lp), nin = ncoef_of(s, lc);
    const int nq = m.ncomp * nrhs;
    const int c0 = s.child_ptr[p], c1 = s.child_ptr[p + 1];
    const int warp = threadIdx.x >> 5;
    double acc[8][2][2];
    warp_acc_zero(acc);
    if (c0 + warp < c1) {  // warp-uniform
        const int ch = s.child[c0 + warp];
        const T *Tk = static_cast<const T *>(s.tr) + s.tr_off[lc * m.nsectors + s.sector[ch]];
        const T *mc = am + s.mom_off[ch] * nrhs;
        warp_mma64x16(nout, nin, nq, [&](int i, int k) -> double { return (double)Tk[i + (int64_t)k * nout]; },
                      [&](int k, int q) -> double { return (double)mc[(int64_t)q * nin + k]; }, acc);
    }
    double *pw = wpart + warp * WARP_TILE;
    warp_acc_store(acc, 64, 16, [&](int i, int q, double v) { pw[q * 64 + i] = v; });
    __syncthreads();
    T *mp = am + s.mom_off[p] * nrhs;
    for (int e = threadIdx.x; e < nout * nq; e += blockDim.x) {
        const int i = e % nout, q = e / nout;
        double v = 0.0;
#pragma unroll
        for (int w = 0; w < 8; ++w) v += wpart[w * WARP_TILE + q * 64 + i];
        narrow(v, mp[(int64_t)q * nout + i]);
    }
}

template <class T>
__global__ void __launch_bounds__(256)
transfer_down_warp_kernel(DMap m, DSide s, const int *__restrict__ nodes, int nnodes,
                          const uint8_t *__restrict__ received, int nrhs, T *__restrict__ dm) {
    const int idx = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (idx >= nnodes) return;  // whole warp; no block barrier
    const int c = nodes[idx];
    const int lc = s.level[c], lp = lc - 1;
    const int par = s.parent[c];
    const int nout = ncoef_of(s, lc), nin = ncoef_of(s, lp);
    const bool acc0 = received[c] != 0;
    const T *Tk = static_cast<const T *>(s.tr) + s.tr_off[lc * m.nsectors + s.sector[c]];
    T *mc = dm + s.mom_off[c] * nrhs;
    const T *mp = dm + s.mom_off[par] * nrhs;
    const int nq = m.ncomp * nrhs;
    double acc[8][2][2];
    warp_acc_zero(acc);
    // stored T is nin x nout (parent x child): op(T)[i, k] = T[k + i * nin]
    warp_mma64x16(nout, nin, nq, [&](int i, int k) -> double { return (double)Tk[k + (int64_t)i * nin]; },
                  [&](int k, int q) -> double { return (double)mp[(int64_t)q * nin + k]; }, acc);
    warp_acc_store(acc, nout, nq, [&](int i, int q, double v) {
        T *dst = &mc[(int64_t)q * nout + i];
        narrow(acc0 ? (double)*dst + v : v, *dst);
    });
}

template <class T>
__global__ void __launch_bounds__(256)
leaf_aggregate_warp_kernel(DMap m, DSide s, const int *__restrict__ leaves, int nleaves, int nrhs,
                           const double *__restrict__ x, int64_t ldx, T *__restrict__ am) {
    const int idx = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (idx >= nleaves) return;  // whole warp; no block barrier
    const int leaf = leaves[idx];
    const int nc = ncoef_of(s, s.level[leaf]);
    const int v0 = s.value_ptr[leaf], nv = s.value_ptr[leaf + 1] - v0;
    const T *C = static_cast<const T *>(s.coll) + s.coll_off[leaf];
    T *mom = am + s.mom_off[leaf] * nrhs;
    const int *vals = s.value + v0;
    for (int c = 0; c < m.ncomp; ++c) {
        const T *Cc = C + (int64_t)c * nc * nv;
        double acc[8][2][2];
        warp_acc_zero(acc);
        warp_mma64x16(nc, nv, nrhs, [&](int i, int k) -> double { return (double)Cc[i + (int64_t)k * nc]; },
                      [&](int k, int q) -> double { return x[(int64_t)q * ldx + vals[k]]; }, acc);
        warp_acc_store(acc, nc, nrhs, [&](int i, int q, double v) { narrow(v, mom[((int64_t)c * nrhs + q) * nc + i]); });
    }
}

// C2 for leaves of any size: the warp takes the leaf's rows 64 at a time (leaves own disjoint
// values, so no two warps write the same entry of y)
template <class T>
__global__ void __launch_bounds__(256)
leaf_disaggregate_warp_kernel(DMap m, DSide s, const int *__restrict__ leaves, int nleaves, int nrhs,
                              const T *__restrict__ dm, double alpha, double beta, bool beta_zero,
                              double *__restrict__ y, int64_t ldy) {
    const int idx = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (idx >= nleaves) return;  // whole warp; no block barrier
    const int leaf = leaves[idx];
    const int nc = ncoef_of(s, s.level[leaf]);
    const int v0 = s.value_ptr[leaf], nv = s.value_ptr[leaf + 1] - v0;
    const T *C = static_cast<const T *>(s.coll) + s.coll_off[leaf];
    const T *mom = dm + s.mom_off[leaf] * nrhs;
    const int *vals = s.value + v0;
    for (int m0 = 0; m0 < nv; m0 += 64) {
        const int mt = min(64, nv - m0);
        double acc[8][2][2];
        warp_acc_zero(acc);
        for (int c = 0; c < m.ncomp; ++c) {
            const T *Cc = C + (int64_t)c * nc * nv;
            const T *mc = mom + (int64_t)c * nrhs * nc;
            // op(C)[i, k] = C[k + i * nc]: the leaf's collection transposed
            warp_mma64x16(mt, nc, nrhs, [&](int i, int k) -> double { return (double)Cc[k + (int64_t)(m0 + i) * nc]; },
                          [&](int k, int q) -> double { return (double)mc[(int64_t)q * nc + k]; }, acc);
        }
        warp_acc_store(acc, mt, nrhs, [&](int i, int q, double v) {
            double *dst = &y[(int64_t)q * ldy + vals[m0 + i]];
            const double w = alpha * v;
            *dst = beta_zero ? w : w + beta * *dst;
        });
    }
}

// Launchers of the warp kernels (real maps only: the complex instantiations are never referenced).
template <class T>
cudaError_t warp_transfer_up(const DMap &m, const DSide &s, const int *nodes, int nnodes, int nrhs, void *am,
                             cudaStream_t st) {
    const size_t wsm = 8 * WARP_TILE * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(transfer_up_warp_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsm);
    if (e == cudaSuccess)
        transfer_up_warp_kernel<T><<<nnodes, 256, wsm, st>>>(m, s, nodes, nrhs, static_cast<T *>(am));
    return e;
}
template <class T>
void warp_transfer_down(const DMap &m, const DSide &s, const int *nodes, int nnodes, const uint8_t *received,
                        int nrhs, void *dm, cudaStream_t st) {
    transfer_down_warp_kernel<T><<<(nnodes + 7) / 8, 256, 0, st>>>(m, s, nodes, nnodes, received, nrhs,
                                                                   static_cast<T *>(dm));
}

// ---------------------------------------------------------------------------------------------
// Toeplitz transforms (modulate_in! / modulate_out!, src/moments/toeplitz/toeplitzmul.jl:290-315).
// Several transforms per CTA, FFT_T threads each, in shared memory. A multidimensional DFT is one
// pass per axis; in a pass each thread owns whole lines along that axis, holds a line in
// registers and writes the transformed line back in place. AbstractFFTs conventions: forward
// e^{-2 pi i jk/n}; inverse e^{+2 pi i jk/n} with 1/n per axis. Axes are at most FFT_NMAX long.
// With `half` set (real maps), only the first n/2 + 1 entries along the first axis are stored; the
// rest follow from Hermitian symmetry S[k] = conj(S[-k]).
// ---------------------------------------------------------------------------------------------
constexpr int FFT_T = 64;
constexpr int FFT_NMAX = 16;

struct TGeom {
    int ts[3];   // padded extents 2s - 1
    int sh[3];   // moment extents s
    int nt, nc;  // padded / moment sizes
    int h0;      // stored extent along the first axis (half or full)
    int slen;    // stored spectrum length
};

// TS > 0: every level's moments are known to be (TS+1)/2-cubes, so the extents are compile-time
// constants and the index arithmetic of the transforms folds to multiplications.
template <int TS = 0>
__device__ __forceinline__ TGeom tgeom(const DSide &s, int lvl, bool half) {
    TGeom g;
    for (int d = 0; d < 3; ++d) {
        g.sh[d] = TS > 0 ? (TS + 1) / 2 : s.shape[3 * lvl + d];
        g.ts[d] = 2 * g.sh[d] - 1;
    }
    g.nt = g.ts[0] * g.ts[1] * g.ts[2];
    g.nc = g.sh[0] * g.sh[1] * g.sh[2];
    g.h0 = half ? g.ts[0] / 2 + 1 : g.ts[0];
    g.slen = g.h0 * g.ts[1] * g.ts[2];
    return g;
}

template <class R, int N>
__device__ __forceinline__ void dft_line(Cx<R> *a, int base, int stride, const Cx<R> *tw, R scale) {
    Cx<R> v[N];
#pragma unroll
    for (int j = 0; j < N; ++j) v[j] = a[base + j * stride];
#pragma unroll
    for (int k = 0; k < N; ++k) {
        Cx<R> acc = v[0];
#pragma unroll
        for (int j = 1; j < N; ++j) acc = acc + v[j] * tw[(j * k) % N];
        a[base + k * stride] = scale * acc;
    }
}

// Padded extents are 2s - 1, hence odd; NMAX bounds the longest line (register footprint).
template <class R, int NMAX>
__device__ __forceinline__ void dft_line_n(int n, Cx<R> *a, int base, int stride, const Cx<R> *tw, R scale) {
    switch (n) {
    case 3: dft_line<R, 3>(a, base, stride, tw, scale); break;
    case 5: dft_line<R, 5>(a, base, stride, tw, scale); break;
    case 7: dft_line<R, 7>(a, base, stride, tw, scale); break;
    case 9: if (NMAX >= 9) dft_line<R, (NMAX >= 9 ? 9 : 3)>(a, base, stride, tw, scale); break;
    case 11: if (NMAX >= 11) dft_line<R, (NMAX >= 11 ? 11 : 3)>(a, base, stride, tw, scale); break;
    case 13: if (NMAX >= 13) dft_line<R, (NMAX >= 13 ? 13 : 3)>(a, base, stride, tw, scale); break;
    case 15: if (NMAX >= 15) dft_line<R, (NMAX >= 15 ? 15 : 3)>(a, base, stride, tw, scale); break;
    default: break;
    }
}

// In-place multidimensional DFT of one transform held by FFT_T threads (tl = thread in group).
// Every thread of the CTA calls this the same number of times (3 barriers), busy or not.
template <class R, int NMAX>
__device__ void dft_group(Cx<R> *a, const TGeom &g, bool inverse, Cx<R> *tw, int tl, bool busy) {
    // twiddles of the three axes: tw[16 * ax + k] = e^{-+2 pi i k / n}
    if (busy)
        for (int e = tl; e < 3 * FFT_NMAX; e += FFT_T) {
            const int ax = e / FFT_NMAX, k = e % FFT_NMAX;
            const int n = g.ts[ax];
            if (k < n) {
                double sv, cv;
                sincospi(2.0 * k / n, &sv, &cv);
                tw[e] = {(R)cv, (R)(inverse ? sv : -sv)};
            }
        }
    __syncthreads();
    for (int ax = 0; ax < 3; ++ax) {
        const int n = g.ts[ax];
        if (busy && n > 1) {
            const int nlines = g.nt / n;
            const R scale = inverse ? (R)1 / (R)n : (R)1;
            for (int l = tl; l < nlines; l += FFT_T) {
                int base, stride;
                if (ax == 0) {
                    base = l * n;
                    stride = 1;
                } else if (ax == 1) {
                    base = (l % g.ts[0]) + g.ts[0] * g.ts[1] * (l / g.ts[0]);
                    stride = g.ts[0];
                } else {
                    base = l;
                    stride = g.ts[0] * g.ts[1];
                }
                dft_line_n<R, NMAX>(n, a, base, stride, tw + FFT_NMAX * ax, scale);
            }
        }
        __syncthreads();
    }
}

// A3: spectrum(node) = F(pad(moment(node)))   (F = fft, or ifft for transpose maps)
template <class T, int NMAX, int TS>
__global__ void __launch_bounds__(256) toeplitz_in_kernel(DMap m, DSide s, const int *__restrict__ nodes, int ntrans, bool inverse,
                                   int nrhs, int maxt, const T *__restrict__ am,
                                   typename ScalarTraits<T>::Complex *__restrict__ as) {
    using S = typename ScalarTraits<T>::Complex;  // stored spectra
    using W = cdouble;                             // transforms run in FP64
    extern __shared__ unsigned char smem_raw[];
    const int grp = threadIdx.x / FFT_T, tl = threadIdx.x % FFT_T, ngrp = blockDim.x / FFT_T;
    W *a = reinterpret_cast<W *>(smem_raw) + (size_t)grp * (maxt + 3 * FFT_NMAX);
    W *tw = a + maxt;
    const int nq = m.ncomp * nrhs;
    const int t = blockIdx.x * ngrp + grp;
    const bool busy = t < ntrans;
    const int node = busy ? nodes[t / nq] : nodes[0];
    const int q = busy ? t % nq : 0;
    const TGeom g = tgeom<TS>(s, s.level[node], m.half_spectrum != 0);
    if (busy) {
        const T *mom = am + s.mom_off[node] * nrhs + (int64_t)q * g.nc;
        for (int e = tl; e < g.nt; e += FFT_T) {
            const int i1 = e % g.ts[0], i2 = (e / g.ts[0]) % g.ts[1], i3 = e / (g.ts[0] * g.ts[1]);
            W v = {0.0, 0.0};
            if (i1 < g.sh[0] && i2 < g.sh[1] && i3 < g.sh[2])
                v = to_cx(wide(mom[i1 + g.sh[0] * (i2 + g.sh[1] * i3)]));
            a[e] = v;
        }
    }
    dft_group<double, NMAX>(a, g, inverse, tw, tl, busy);
    if (busy) {
        S *spec = as + s.spec_off[node] * nrhs + (int64_t)q * g.slen;
        for (int e = tl; e < g.slen; e += FFT_T) {
            const int k1 = e % g.h0, r = e / g.h0;
            narrow(a[k1 + g.ts[0] * r], spec[e]);
        }
    }
}

// B3: moment(node) = corner(F^-1(spectrum(node)))   (overwrite)
template <class T, int NMAX, int TS>
__global__ void __launch_bounds__(256) toeplitz_out_kernel(DMap m, DSide s, const int *__restrict__ nodes, int ntrans, bool inverse,
                                    int nrhs, int maxt,
                                    const typename ScalarTraits<T>::Complex *__restrict__ ds,
                                    T *__restrict__ dm) {
    using S = typename ScalarTraits<T>::Complex;  // stored spectra
    using W = cdouble;                             // transforms run in FP64
    extern __shared__ unsigned char smem_raw[];
    const int grp = threadIdx.x / FFT_T, tl = threadIdx.x % FFT_T, ngrp = blockDim.x / FFT_T;
    W *a = reinterpret_cast<W *>(smem_raw) + (size_t)grp * (maxt + 3 * FFT_NMAX);
    W *tw = a + maxt;
    const int nq = m.ncomp * nrhs;
    const int t = blockIdx.x * ngrp + grp;
    const bool busy = t < ntrans;
    const int node = busy ? nodes[t / nq] : nodes[0];
    const int q = busy ? t % nq : 0;
    const TGeom g = tgeom<TS>(s, s.level[node], m.half_spectrum != 0);
    if (busy) {
        const S *spec = ds + s.spec_off[node] * nrhs + (int64_t)q * g.slen;
        for (int e = tl; e < g.nt; e += FFT_T) {
            const int k1 = e % g.ts[0], r = e / g.ts[0];
            if (k1 < g.h0) {
                a[e] = wide(spec[k1 + g.h0 * r]);
            } else {
                const int k2 = r % g.ts[1], k3 = r / g.ts[1];
                const int m1 = g.ts[0] - k1, m2 = (g.ts[1] - k2) % g.ts[1], m3 = (g.ts[2] - k3) % g.ts[2];
                a[e] = conjg(wide(spec[m1 + g.h0 * (m2 + g.ts[1] * m3)]));
            }
        }
    }
    dft_group<double, NMAX>(a, g, inverse, tw, tl, busy);
    if (busy) {
        T *mom = dm + s.mom_off[node] * nrhs + (int64_t)q * g.nc;
        for (int e = tl; e < g.nc; e += FFT_T) {
            const int i1 = e % g.sh[0], i2 = (e / g.sh[0]) % g.sh[1], i3 = e / (g.sh[0] * g.sh[1]);
            from_cx(a[i1 + g.ts[0] * (i2 + g.ts[1] * i3)], mom[e]);
        }
    }
}

// Pruned transforms of real maps with 4-point cube moments (padded 7^3, half spectra 4 x 7 x 7):
// the zero padding and the Hermitian half are never computed. In: the moment (4^3 reals) is
// transformed along axis 0 into the 4 stored frequencies only (4^3 outputs), then along axis 1
// (4 x 7 x 4) and axis 2 (4 x 7 x 7), each output a 4-term sum over the non-zero inputs; 1,488
// complex multiply-adds against 7,203 for the three full line passes. Out: the inverse pass runs
// axis 2 then axis 1 into the 4^3 corner only, and axis 0 rebuilds the real corner values from the
// stored half, x[i] = Re Q[0] + 2 Re sum_{k=1..3} Q[k] w^{ki} (Q is Hermitian along axis 0 once
// axes 1 and 2 are back in space). FP64 arithmetic; one transform per 64 threads.
// ---------------------------------------------------------------------------------------------
constexpr int PR_T = 64;   // threads per transform
constexpr int PR_G = 4;    // transforms per CTA

__device__ __forceinline__ void pr_twiddles(cdouble *tw, bool inverse) {
    if (threadIdx.x < 7) {
        double sv, cv;
        sincospi(2.0 * threadIdx.x / 7.0, &sv, &cv);
        tw[threadIdx.x] = {cv, inverse ? sv : -sv};
    }
}

template <class T>
__global__ void __launch_bounds__(PR_T * PR_G)
toeplitz_in_cube4_real_kernel(DSide s, const int *__restrict__ nodes, int ntrans, bool inverse, int nq,
                              int nrhs, const T *__restrict__ am,
                              typename ScalarTraits<T>::Complex *__restrict__ as) {
    using S = typename ScalarTraits<T>::Complex;
    __shared__ cdouble tw[7];
    __shared__ double mom[PR_G][64];
    __shared__ cdouble A[PR_G][64];   // [k1 < 4][i2 < 4][i3 < 4]
    __shared__ cdouble B[PR_G][112];  // [k1 < 4][k2 < 7][i3 < 4]
    const int grp = threadIdx.x / PR_T, tl = threadIdx.x % PR_T;
    const int t = blockIdx.x * PR_G + grp;
    const bool busy = t < ntrans;
    const int node = busy ? nodes[t / nq] : nodes[0];
    const int q = busy ? t % nq : 0;
    pr_twiddles(tw, inverse);
    if (busy) mom[grp][tl] = (double)am[s.mom_off[node] * nrhs + (int64_t)q * 64 + tl];
    __syncthreads();
    {  // axis 0: real inputs i1 < 4, stored frequencies k1 < 4
        const int k1 = tl & 3, r = tl >> 2;
        cdouble a = {0.0, 0.0};
#pragma unroll
        for (int i1 = 0; i1 < 4; ++i1) a = a + mom[grp][i1 + 4 * r] * tw[(k1 * i1) % 7];
        A[grp][tl] = a;
    }
    __syncthreads();
    for (int o = tl; o < 112; o += PR_T) {  // axis 1: inputs i2 < 4, all k2 < 7
        const int k1 = o & 3, k2 = (o >> 2) % 7, i3 = o / 28;
        cdouble b = {0.0, 0.0};
#pragma unroll
        for (int i2 = 0; i2 < 4; ++i2) b = b + A[grp][k1 + 4 * (i2 + 4 * i3)] * tw[(k2 * i2) % 7];
        B[grp][o] = b;
    }
    __syncthreads();
    if (busy) {  // axis 2: inputs i3 < 4, all k3 < 7; stored as [k1][k2][k3]
        S *spec = as + s.spec_off[node] * nrhs + (int64_t)q * 196;
        const double sc = inverse ? 1.0 / 343.0 : 1.0;
        for (int o = tl; o < 196; o += PR_T) {
            const int k12 = o % 28, k3 = o / 28;
            cdouble c = {0.0, 0.0};
#pragma unroll
            for (int i3 = 0; i3 < 4; ++i3) c = c + B[grp][k12 + 28 * i3] * tw[(k3 * i3) % 7];
            narrow(sc * c, spec[o]);
        }
    }
}

template <class T>
__global__ void __launch_bounds__(PR_T * PR_G)
toeplitz_out_cube4_real_kernel(DSide s, const int *__restrict__ nodes, int ntrans, bool inverse, int nq,
                               int nrhs, const typename ScalarTraits<T>::Complex *__restrict__ ds,
                               T *__restrict__ dm) {
    __shared__ cdouble tw[7];
    __shared__ cdouble X[PR_G][196];  // stored half spectrum [k1 < 4][k2 < 7][k3 < 7]
    __shared__ cdouble P[PR_G][112];  // [k1 < 4][k2 < 7][i3 < 4]
    __shared__ cdouble Q[PR_G][64];   // [k1 < 4][i2 < 4][i3 < 4]
    const int grp = threadIdx.x / PR_T, tl = threadIdx.x % PR_T;
    const int t = blockIdx.x * PR_G + grp;
    const bool busy = t < ntrans;
    const int node = busy ? nodes[t / nq] : nodes[0];
    const int q = busy ? t % nq : 0;
    pr_twiddles(tw, inverse);
    if (busy) {
        const auto *spec = ds + s.spec_off[node] * nrhs + (int64_t)q * 196;
        for (int o = tl; o < 196; o += PR_T) X[grp][o] = wide(spec[o]);
    }
    __syncthreads();
    for (int o = tl; o < 112; o += PR_T) {  // axis 2 back to i3 < 4
        const int k12 = o % 28, i3 = o / 28;
        cdouble p = {0.0, 0.0};
#pragma unroll
        for (int k3 = 0; k3 < 7; ++k3) p = p + X[grp][k12 + 28 * k3] * tw[(k3 * i3) % 7];
        P[grp][o] = p;
    }
    __syncthreads();
    {  // axis 1 back to i2 < 4
        const int k1 = tl & 3, i2 = (tl >> 2) & 3, i3 = tl >> 4;
        cdouble v = {0.0, 0.0};
#pragma unroll
        for (int k2 = 0; k2 < 7; ++k2) v = v + P[grp][k1 + 4 * (k2 + 7 * i3)] * tw[(k2 * i2) % 7];
        Q[grp][tl] = v;
    }
    __syncthreads();
    if (busy) {  // axis 0 from the Hermitian half, real corner i1 < 4
        const int i1 = tl & 3, r = tl >> 2;
        const cdouble *qv = &Q[grp][4 * r];
        double x = qv[0].x;
#pragma unroll
        for (int k1 = 1; k1 < 4; ++k1) {
            const cdouble w = tw[(k1 * i1) % 7];
            x += 2.0 * (qv[k1].x * w.x - qv[k1].y * w.y);
        }
        const double sc = inverse ? 1.0 / 343.0 : 1.0;
        narrow(sc * x, dm[s.mom_off[node] * nrhs + (int64_t)q * 64 + tl]);
    }
}

// ---------------------------------------------------------------------------------------------
// B1/B2: l_r = sum over pairs of op(B_key) m_t (dense), d .* m_t (diagonal), or, for Toeplitz,
// S_r = sum K_key .* S_t on the spectra. op: identity / transpose / adjoint by map orientation
// (src/farinteractions/i2otranslations/i2oprotocol.jl:87-92, i2otranslationcollection.jl:367-495,
// toeplitzi2ocollection.jl:110-193). The first pair overwrites.
// ---------------------------------------------------------------------------------------------
template <class T, bool MMA>
__global__ void __launch_bounds__(512) i2o_kernel(DMap m, DSide r, DSide t, const int *__restrict__ nodes, int mode,
                           int nrhs, const T *__restrict__ am, T *__restrict__ dm,
                           const typename ScalarTraits<T>::Complex *__restrict__ as,
                           typename ScalarTraits<T>::Complex *__restrict__ ds) {
    using S = typename ScalarTraits<T>::Complex;
    using A = typename ScalarTraits<T>::Acc;
    const int node = nodes[blockIdx.x];
    const int p0 = r.i2o_ptr[node], p1 = r.i2o_ptr[node + 1];
    const int lvl = r.level[node];
    const int nc = ncoef_of(r, lvl);
    const int nq = m.ncomp * nrhs;
    const bool adj = (mode == H2B_ADJOINT);
    // r.pair_src[p]: the source's moment (or spectrum) offset per unit rhs; r.pair_cpl[p]: the
    // coupling's element offset -- one load each per pair, no chained index lookups
    if (m.coupling_kind == H2B_COUPLING_TOEPLITZ) {
        // each kernel value is loaded once and applied to up to QB right-hand sides
        constexpr int QB = 8;
        const int nt = tgeom<>(r, lvl, m.half_spectrum != 0).slen;
        S *out = ds + r.spec_off[node] * nrhs;
        const S *K0 = static_cast<const S *>(m.cpl);
        for (int q0 = 0; q0 < nq; q0 += QB) {
            const int qc = min(QB, nq - q0);
            for (int e = threadIdx.x; e < nt; e += blockDim.x) {
                if (qc == 1) {
                    cdouble acc = {0.0, 0.0};
                    int p = p0;
                    for (; p + 4 <= p1; p += 4) {
                        S kv[4], iv[4];
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            kv[u] = K0[r.pair_cpl[p + u] + e];
                            iv[u] = as[r.pair_src[p + u] * nrhs + (int64_t)q0 * nt + e];
                        }
#pragma unroll
                        for (int u = 0; u < 4; ++u) acc = acc + wide(cj(kv[u], adj)) * wide(iv[u]);
                    }
                    for (; p < p1; ++p)
                        acc = acc + wide(cj(K0[r.pair_cpl[p] + e], adj)) *
                                        wide(as[r.pair_src[p] * nrhs + (int64_t)q0 * nt + e]);
                    narrow(acc, out[(int64_t)q0 * nt + e]);
                } else {
                    cdouble acc[QB];
#pragma unroll
                    for (int q = 0; q < QB; ++q) acc[q] = cdouble{0.0, 0.0};
                    for (int p = p0; p < p1; ++p) {
                        const cdouble kv = wide(cj(K0[r.pair_cpl[p] + e], adj));
                        const S *in = as + r.pair_src[p] * nrhs + (int64_t)q0 * nt + e;
#pragma unroll
                        for (int q = 0; q < QB; ++q)
                            if (q < qc) acc[q] = acc[q] + kv * wide(in[(int64_t)q * nt]);
                    }
#pragma unroll
                    for (int q = 0; q < QB; ++q)
                        if (q < qc) narrow(acc[q], out[(int64_t)(q0 + q) * nt + e]);
                }
            }
        }
        return;
    }
    T *out = dm + r.mom_off[node] * nrhs;
    const T *B0 = static_cast<const T *>(m.cpl);
    if (m.coupling_kind == H2B_COUPLING_DIAGONAL) {
        for (int q = 0; q < nq; ++q)
            for (int a = threadIdx.x; a < nc; a += blockDim.x) {
                A acc = sc_zero<A>();
                for (int p = p0; p < p1; ++p) {
                    const T *D = B0 + r.pair_cpl[p];
                    acc = acc + wide(cj(D[a], adj)) * wide(am[r.pair_src[p] * nrhs + (int64_t)q * nc + a]);
                }
                narrow(acc, out[(int64_t)q * nc + a]);
            }
        return;
    }
    // dense: out (nc x nq) = sum over pairs of op(B) X_src, all right-hand sides per pass, on
    // the FP64 tensor cores (tile_gemm_mma_l; the CTA has the 8 warps its tiling needs)
    extern __shared__ unsigned char smem_raw[];
    A *Ms = reinterpret_cast<A *>(smem_raw), *Xs = Ms + TG_M * TG_LD;
    for (int q0 = 0; q0 < nq; q0 += TG_Q) {
        const int nqc = min(TG_Q, nq - q0);
        for (int m0 = 0; m0 < nc; m0 += TG_M) {
            const int mt = min(TG_M, nc - m0);
            // one right-hand side (MMA false): FMA tile (an MMA would idle 7 of its 8 columns)
            MmaAcc<A> acc;
            acc.zero();
            A accf[TG_O];
            tile_zero(accf);
            for (int p = p0; p < p1; ++p) {
                const int snc = ncoef_of(t, t.level[r.i2o_src[p]]);
                const T *B = B0 + r.pair_cpl[p];
                const T *X = am + r.pair_src[p] * nrhs;
                const int64_t ps = r.pair_perm ? r.pair_perm[p] : -1;
                auto prod = [&](bool kfast, auto mload, auto xload) {
                    if constexpr (!MMA) tile_gemm_l(kfast, m0, mt, snc, nqc, mload, xload, Ms, Xs, accf);
                    else tile_gemm_mma_l(kfast, m0, mt, snc, nqc, mload, xload, Ms, Xs, acc);
                };
                auto xl = [&](int k, int q) -> A { return wide(X[(int64_t)(q0 + q) * snc + k]); };
                if (ps < 0 && mode == H2B_FORWARD) {
                    // forward: block (r, t) is nc x snc
                    prod(false, [&](int i, int k) -> A { return wide(cj(B[i + (int64_t)k * nc], adj)); }, xl);
                } else if (ps < 0) {
                    // transposed: block (t, r) is snc x nc
                    prod(true, [&](int i, int k) -> A { return wide(cj(B[k + (int64_t)i * snc], adj)); }, xl);
                } else if (mode == H2B_FORWARD) {
                    // t[rp[i], cp[j]] = M[i, j]: out[i] += sum_j M[rp^-1[i], j] x[cp[j]]
                    // (gather / canonical product / scatter of symmetryreduceddense.jl:84-95,
                    // with the scatter folded into the row index)
                    const int *ri = m.perm + ps + nc, *cp = m.perm + ps + 2 * nc;
                    prod(false, [&](int i, int k) -> A { return wide(cj(B[ri[i] + (int64_t)k * nc], adj)); },
                         [&](int k, int q) -> A { return wide(X[(int64_t)(q0 + q) * snc + cp[k]]); });
                } else {
                    // transposed / adjoint: out[j] += sum_i op(M)[cp^-1[j], i] x[rp[i]]
                    const int *rp = m.perm + ps, *ci = m.perm + ps + 3 * snc;
                    prod(true, [&](int i, int k) -> A { return wide(cj(B[k + (int64_t)ci[i] * snc], adj)); },
                         [&](int k, int q) -> A { return wide(X[(int64_t)(q0 + q) * snc + rp[k]]); });
                }
            }
            if constexpr (!MMA) {
#pragma unroll
                for (int j = 0; j < TG_O; ++j) {
                    const int o = threadIdx.x + j * blockDim.x;
                    if (o < mt * nqc) narrow(accf[j], out[(int64_t)(q0 + o / mt) * nc + m0 + o % mt]);
                }
            } else {
                mma_store(acc, mt, nqc, [&](int i, int q, A v) { narrow(v, out[(int64_t)(q0 + q) * nc + m0 + i]); });
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// B1 for few right-hand sides, grouped by stored block (GroupTiles). One CTA per chunk of receiving
// nodes of one level. For each run of pairs reading one stored block the block is staged in 64 x 32
// pieces (cp.async, two stages: the next chunk's copies fly while the tensor cores work on this
// one), each piece applied to up to GT_NB column blocks of TG_Q columns (pairs x right-hand sides)
// on the FP64 tensor cores; each pair's symmetry permutation moves into the gather of its moments
// (column permutation) and the row its products land on (row permutation), the canonical form of
// symmetryreduceddense.jl:84-95. Products add into the chunk's sums in shared memory; the tiles
// follow one another behind the tile product's block barriers, and within a tile every pair has
// its own receiver, so no two threads add into one sum at once. The sums are written once at the
// end (overwriting each receiving node's I2O output, as the per-node kernels do).
// ---------------------------------------------------------------------------------------------
// column blocks of TG_Q columns held at once per staged piece of a block (their FP64 fragments:
// 4 doubles per block and lane for real sums, 8 for complex)
template <class A> constexpr int gt_nb() { return sizeof(A) == 16 ? 4 : 8; }

// element copy global -> shared (cp.async); ok = false writes zeros and reads nothing
template <int EB>
__device__ __forceinline__ void cp_async_elem(void *dst, const void *src, bool ok) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src), "n"(EB), "r"(ok ? EB : 0)
                 : "memory");
}

template <class T>
__global__ void __launch_bounds__(256)
i2o_grouped_kernel(DMap m, DSide r, DSide t, GroupTiles gt, int mode, int nrhs, int maxcoef,
                   const T *__restrict__ am, T *__restrict__ dm) {
    using A = typename ScalarTraits<T>::Acc;
    constexpr int GT_NB = gt_nb<A>();
    constexpr int EB = sizeof(T);
    constexpr int MS = TG_M * TG_LD, XS = GT_NB * TG_K * TG_Q;  // one stage of the block / moments
    extern __shared__ unsigned char smem_raw[];
    // the receivers' FP64 sums, then two stages of the block piece and the moments in the storage
    // type (copied with cp.async one chunk ahead, widened when the products read them)
    const int nq = m.ncomp * nrhs;
    A *Sum = reinterpret_cast<A *>(smem_raw);
    T *Mst = reinterpret_cast<T *>(Sum + GT_R * nq * maxcoef);
    T *Xst = Mst + 2 * MS;
    // per pair of the current run (slot b * TG_Q + j: pair j of column block b): its moments' offset,
    // its permutation set (-1: none) and its receiver's position in the chunk
    __shared__ int64_t run_src[GT_NB * TG_Q], run_perm[GT_NB * TG_Q];
    __shared__ int run_slot[GT_NB * TG_Q];
    const int ch = blockIdx.x;
    const int r0 = gt.chunk_ptr[ch], nr = gt.chunk_ptr[ch + 1] - r0;
    const int nc = ncoef_of(r, r.level[gt.rcv[r0]]);
    const bool fwd = mode == H2B_FORWARD, adj = mode == H2B_ADJOINT;
    const T *B0 = static_cast<const T *>(m.cpl);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g4 = lane >> 2, t4 = lane & 3;
    for (int o = threadIdx.x; o < nr * nq * nc; o += blockDim.x) Sum[o] = A{};
    const int pq = TG_Q / nq;  // pairs per column block
    const int t_end = gt.tile_ptr[ch + 1];
    for (int tl = gt.tile_ptr[ch]; tl < t_end;) {
        // a run of tiles reading one stored block, cut into column blocks of pq pairs (at most
        // GT_NB): every block holds pairs of distinct receivers, since each tile does
        const int pf = gt.pair[gt.tile_pp[tl]];
        const int64_t key = r.pair_cpl[pf];
        int bs[GT_NB], bn[GT_NB], nb = 0;  // first pair and pair count of each block
        int tl2 = tl;
        while (tl2 < t_end && r.pair_cpl[gt.pair[gt.tile_pp[tl2]]] == key) {
            const int e0 = gt.tile_pp[tl2], e1 = gt.tile_pp[tl2 + 1];
            const int need = (e1 - e0 + pq - 1) / pq;
            if (nb + need > GT_NB) break;
            for (int e = e0; e < e1; e += pq) {
                bs[nb] = e;
                bn[nb] = min(pq, e1 - e);
                ++nb;
            }
            ++tl2;
        }
        tl = tl2;
        const int snc = ncoef_of(t, t.level[r.i2o_src[pf]]);
        const T *B = B0 + key;  // the run's stored block
        __syncthreads();  // the previous run's stores have read its pair table
        for (int j = threadIdx.x; j < GT_NB * TG_Q; j += blockDim.x) {
            const int b = j / TG_Q, jj = j % TG_Q;
            if (b < nb && jj < bn[b]) {
                const int e = bs[b] + jj;
                const int p = gt.pair[e];
                run_src[j] = r.pair_src[p] * nrhs;
                run_perm[j] = r.pair_perm ? r.pair_perm[p] : -1;
                run_slot[j] = gt.slot[e];
            }
        }
        __syncthreads();
        const int nk = (snc + TG_K - 1) / TG_K;
        for (int m0 = 0; m0 < nc; m0 += TG_M) {
            const int mt = min(TG_M, nc - m0);
            // chunk kc's copies into stage kc & 1: the block piece (forward reads the stored (r, t)
            // block nc x snc down its columns, transposed orientations the stored (t, r) block
            // snc x nc along k) and each column block's moments, read through the pair's column
            // permutation (forward) or row permutation (transposed); past the block: zeros
            auto issue = [&](int kc) {
                const int k0 = kc * TG_K, kv = min(TG_K, snc - k0);
                T *ms = Mst + (kc & 1) * MS;
                if (fwd) {
                    for (int idx = threadIdx.x; idx < mt * TG_K; idx += blockDim.x) {
                        const int i = idx % mt, k = idx / mt;
                        const bool ok = k < kv;
                        cp_async_elem<EB>(ms + i * TG_LD + k, ok ? B + m0 + i + (int64_t)(k0 + k) * nc : B, ok);
                    }
                } else {
                    for (int idx = threadIdx.x; idx < mt * TG_K; idx += blockDim.x) {
                        const int k = idx % TG_K, i = idx / TG_K;
                        const bool ok = k < kv;
                        cp_async_elem<EB>(ms + i * TG_LD + k, ok ? B + k0 + k + (int64_t)(m0 + i) * snc : B, ok);
                    }
                }
                T *xst = Xst + (kc & 1) * XS;
                for (int b = 0; b < nb; ++b) {
                    const int ncol = bn[b] * nq;
                    T *xs = xst + b * TG_K * TG_Q;
                    for (int idx = threadIdx.x; idx < TG_K * ncol; idx += blockDim.x) {
                        const int k = idx % TG_K, c = idx / TG_K;
                        const int j = b * TG_Q + c / nq;
                        const bool ok = k < kv;
                        const int64_t ps = run_perm[j];
                        const int kk = !ok ? 0 : (ps < 0 ? k0 + k : m.perm[ps + (fwd ? 2 * snc : 0) + k0 + k]);
                        cp_async_elem<EB>(xs + k * TG_Q + c, am + run_src[j] + (int64_t)(c % nq) * snc + kk, ok);
                    }
                }
            };
            MmaAcc<A> acc[GT_NB];
#pragma unroll
            for (int b = 0; b < GT_NB; ++b) acc[b].zero();
            issue(0);
            asm volatile("cp.async.commit_group;" ::: "memory");
            for (int kc = 0; kc < nk; ++kc) {
                if (kc + 1 < nk) issue(kc + 1);  // its stage was last read before the barrier below
                asm volatile("cp.async.commit_group;" ::: "memory");
                asm volatile("cp.async.wait_group 1;" ::: "memory");  // this thread's chunk kc
                __syncthreads();                                      // ... and everyone's
                if (8 * warp < mt) {
                    const T *mrow = Mst + (kc & 1) * MS + (8 * warp + g4) * TG_LD + t4;
                    const T *xst = Xst + (kc & 1) * XS;
#pragma unroll
                    for (int k = 0; k < TG_K; k += 4) {
                        const A a = wide(cj(mrow[k], adj));
#pragma unroll
                        for (int b = 0; b < GT_NB; ++b) {
                            if (b < nb) {
                                const T *xcol = xst + b * TG_K * TG_Q + (t4 + k) * TG_Q + g4;
                                const A bb[2] = {wide(xcol[0]), wide(xcol[8])};
                                acc[b].step(a, bb);
                            }
                        }
                    }
                }
                __syncthreads();  // stage kc & 1 is free for chunk kc + 2
            }
            // the blocks' products into the receivers' sums, one block after another
#pragma unroll
            for (int b = 0; b < GT_NB; ++b) {
                if (b < nb) {
                    __syncthreads();
                    mma_store(acc[b], mt, bn[b] * nq, [&](int i, int c, A v) {
                        const int j = b * TG_Q + c / nq;
                        const int64_t ps = run_perm[j];
                        const int row = ps < 0 ? m0 + i : m.perm[ps + (fwd ? 0 : 2 * nc) + m0 + i];
                        A &sum = Sum[(run_slot[j] * nq + c % nq) * nc + row];
                        sum = sum + v;
                    });
                }
            }
        }
    }
    __syncthreads();
    for (int o = threadIdx.x; o < nr * nq * nc; o += blockDim.x) {
        const int ls = o / (nq * nc);
        narrow(Sum[o], dm[r.mom_off[gt.rcv[r0 + ls]] * nrhs + o % (nq * nc)]);
    }
}

// ---------------------------------------------------------------------------------------------
// B2 by sibling groups: the Toeplitz I2O of the receiving children of one parent together. One CTA
// per (group, block of right-hand sides), one thread per stored frequency. The CTA walks the union
// of the siblings' sources once; each source spectrum value is loaded once and applied from
// registers to every sibling translating from it, with that pair's kernel value (loaded through
// L1). Per complex multiply-add this moves one kernel value per QB right-hand sides and one source
// value per group instead of one of each per pair.
// ---------------------------------------------------------------------------------------------
// SL child slots per thread (8: one thread per frequency; 4: two threads per frequency, half
// the accumulators), U source entries per step with every load issued before the arithmetic.
template <class T, int QB, int SL, int U>
__global__ void __launch_bounds__(512)
i2o_sibling_kernel(DMap m, DSide r, SibGroups g, int mode, int nrhs, int et,
                   const typename ScalarTraits<T>::Complex *__restrict__ as,
                   typename ScalarTraits<T>::Complex *__restrict__ ds) {
    using S = typename ScalarTraits<T>::Complex;
    const int gi = blockIdx.x;
    const int q0 = blockIdx.y * QB;
    const int nq = m.ncomp * nrhs;
    const int e = threadIdx.x % et, s0 = (threadIdx.x / et) * SL;  // frequency, first slot
    const int slen = g.slen[gi];
    if (e >= slen) return;  // no barriers below
    const bool adj = mode == H2B_ADJOINT;
    const S *K0 = static_cast<const S *>(m.cpl);
    const int k0 = g.ptr[gi], k1 = g.ptr[gi + 1];
    // accumulated in the storage type: FP64 in the FP64 form; FP32 in the FP32 form, whose sums of
    // at most one interaction list (189 pairs in a uniform tree) per frequency keep the product
    // within 3.2e-7 of the FP64 one on the benchmark map (2.2e-7 with FP64 sums)
    S acc[SL][QB];
#pragma unroll
    for (int sl = 0; sl < SL; ++sl)
#pragma unroll
        for (int q = 0; q < QB; ++q) acc[sl][q] = S{};
    for (int k = k0; k < k1; k += U) {
        S sv[U][QB];
        int ko[U][SL];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const bool ok = k + u < k1;
            const int *kof = g.kof + (int64_t)(ok ? k + u : k) * 8 + s0;
#pragma unroll
            for (int sl = 0; sl < SL; ++sl) ko[u][sl] = ok ? kof[sl] : -1;
            const S *sp = as + g.src_off[ok ? k + u : k] * nrhs + (int64_t)q0 * slen + e;
#pragma unroll
            for (int q = 0; q < QB; ++q) sv[u][q] = q0 + q < nq ? sp[(int64_t)q * slen] : S{};
        }
        S kvs[U][SL];
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int sl = 0; sl < SL; ++sl) kvs[u][sl] = ko[u][sl] >= 0 ? K0[ko[u][sl] + e] : S{};
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int sl = 0; sl < SL; ++sl) {
                if (ko[u][sl] >= 0) {
                    const S kv = cj(kvs[u][sl], adj);
#pragma unroll
                    for (int q = 0; q < QB; ++q) acc[sl][q] = acc[sl][q] + kv * sv[u][q];
                }
            }
    }
#pragma unroll
    for (int sl = 0; sl < SL; ++sl) {
        const int rv = g.recv[gi * 8 + s0 + sl];
        if (rv < 0) continue;
        S *out = ds + r.spec_off[rv] * nrhs + (int64_t)q0 * slen + e;
#pragma unroll
        for (int q = 0; q < QB; ++q)
            if (q0 + q < nq) out[(int64_t)q * slen] = acc[sl][q];
    }
}

// The sibling-group product on the FP64 tensor cores, for blocks of right-hand sides. Per (group,
// stored frequency f) the eight receiving slots and the right-hand sides form one complex product
// out[slot][q] = sum over the group's sources j of K_f(slot, j) S_f(j, q); in real form
//   Re out = sum_j (Kr Sr - Ki Si),  Im out = sum_j (Ki Sr + Kr Si),
// i.e. two 8-row products (Re and Im rows) over K = (source, Re/Im part of S). One warp per
// frequency: each mma.sync m8n8k4 covers two sources; lane (g, t) holds A = K_f(slot g, source
// t / 2) in the Re or Im row form for part t % 2, and B = that part of S_f(source t / 2, rhs g).
// Sums stay in FP64 fragments (8 doubles per lane for 16 right-hand sides), so a warp holds little
// state and many warps stay resident; FP32 spectra and kernel values widen on load.
template <class S, int NTQ>
__global__ void __launch_bounds__(256)
i2o_sibling_dmma_kernel(DMap m, DSide r, SibGroups g, int mode, int nrhs, const S *__restrict__ as,
                        S *__restrict__ ds) {
    const int gi = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int e = blockIdx.y * 8 + warp;  // stored frequency
    const int slen = g.slen[gi];
    if (e >= slen) return;  // whole warp; no block barrier
    const int nq = m.ncomp * nrhs;
    const int q0 = blockIdx.z * 8 * NTQ;
    const int g4 = lane >> 2, t4 = lane & 3;
    const bool part_re = (t4 & 1) == 0;
    const double csign = mode == H2B_ADJOINT ? -1.0 : 1.0;  // adjoint maps conjugate the kernel
    const S *K0 = static_cast<const S *>(m.cpl);
    const int k0 = g.ptr[gi], k1 = g.ptr[gi + 1];
    double cre[NTQ][2], cim[NTQ][2];
#pragma unroll
    for (int u = 0; u < NTQ; ++u) cre[u][0] = cre[u][1] = cim[u][0] = cim[u][1] = 0.0;
#pragma unroll 2
    for (int k = k0; k < k1; k += 2) {
        const int src = k + (t4 >> 1);
        const bool ok = src < k1;
        const int ko = ok ? g.kof[(int64_t)src * 8 + g4] : -1;
        double kr = 0.0, ki = 0.0;
        if (ko >= 0) {
            const S kv = K0[ko + e];
            kr = kv.x;
            ki = csign * kv.y;
        }
        const double are = part_re ? kr : -ki, aim = part_re ? ki : kr;
        const S *sp = as + (ok ? g.src_off[src] : g.src_off[k0]) * nrhs + (int64_t)q0 * slen + e;
#pragma unroll
        for (int u = 0; u < NTQ; ++u) {
            const int q = 8 * u + g4;
            double b = 0.0;
            if (ok && q0 + q < nq) {
                const S x = sp[(int64_t)q * slen];
                b = part_re ? (double)x.x : (double)x.y;
            }
            dmma8(cre[u], are, b);
            dmma8(cim[u], aim, b);
        }
    }
    // C fragment: slot g4, right-hand sides 8u + 2 t4 + h
    const int rv = g.recv[gi * 8 + g4];
    if (rv < 0) return;
    S *out = ds + r.spec_off[rv] * nrhs + (int64_t)q0 * slen + e;
#pragma unroll
    for (int u = 0; u < NTQ; ++u)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int q = 8 * u + 2 * t4 + h;
            if (q0 + q < nq) {
                S v;
                v.x = cre[u][h];
                v.y = cim[u][h];
                out[(int64_t)q * slen] = v;
            }
        }
}

// The same product with one thread per (child slot, stored frequency): a warp covers 8 slots x
// 4 frequencies, a CTA 32 frequencies of one group and QB right-hand sides. Each thread loads its
// pair's kernel value once per source entry and applies it to QB source values (loaded by the 8
// slot threads of a frequency at once, one L1 line); its accumulators are only QB wide, so QB can
// cover a whole 16-RHS block, and 8x more threads than the frequency-per-thread form keep more
// loads in flight. Entries are unrolled by U.
template <class T, int QB, int U>
__global__ void __launch_bounds__(256)
i2o_slot_kernel(DMap m, DSide r, SibGroups g, int mode, int nrhs,
                const typename ScalarTraits<T>::Complex *__restrict__ as,
                typename ScalarTraits<T>::Complex *__restrict__ ds) {
    using S = typename ScalarTraits<T>::Complex;
    const int gi = blockIdx.x;
    const int q0 = blockIdx.z * QB;
    const int nq = m.ncomp * nrhs;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int sl = lane >> 2;
    const int e = blockIdx.y * 32 + warp * 4 + (lane & 3);
    const int slen = g.slen[gi];
    const int rv = g.recv[gi * 8 + sl];
    if (e >= slen || rv < 0) return;  // no barriers below
    const bool adj = mode == H2B_ADJOINT;
    const S *K0 = static_cast<const S *>(m.cpl);
    const int k0 = g.ptr[gi], k1 = g.ptr[gi + 1];
    S acc[QB];
#pragma unroll
    for (int q = 0; q < QB; ++q) acc[q] = S{};
    const int qn = min(QB, nq - q0);
    for (int k = k0; k < k1; k += U) {
        int ko[U];
        const S *sp[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const bool ok = k + u < k1;
            ko[u] = ok ? g.kof[(int64_t)(k + u) * 8 + sl] : -1;
            sp[u] = as + g.src_off[ok ? k + u : k] * nrhs + (int64_t)q0 * slen + e;
        }
        S kv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) kv[u] = ko[u] >= 0 ? cj(K0[ko[u] + e], adj) : S{};
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (ko[u] < 0) continue;
#pragma unroll
            for (int q = 0; q < QB; ++q)
                if (q < qn) acc[q] = acc[q] + kv[u] * sp[u][(int64_t)q * slen];
        }
    }
    S *out = ds + r.spec_off[rv] * nrhs + (int64_t)q0 * slen + e;
#pragma unroll
    for (int q = 0; q < QB; ++q)
        if (q < qn) out[(int64_t)q * slen] = acc[q];
}

// ---------------------------------------------------------------------------------------------
// C1: l_c = [l_c +] op(T_{level(c), sector(c)}) l_parent, op = transpose (adjoint for adjoint maps)
// ---------------------------------------------------------------------------------------------
template <class T, bool MMA>
__global__ void transfer_down_kernel(DMap m, DSide s, const int *__restrict__ nodes,
                                     const uint8_t *__restrict__ received, bool conjt, int nrhs,
                                     T *__restrict__ dm) {
    using A = typename ScalarTraits<T>::Acc;
    extern __shared__ unsigned char smem_raw[];
    A *sm = reinterpret_cast<A *>(smem_raw);
    const int c = nodes[blockIdx.x];
    const int lc = s.level[c], lp = lc - 1;
    const int par = s.parent[c];
    const int nout = ncoef_of(s, lc), nin = ncoef_of(s, lp);
    const bool acc0 = received[c] != 0;
    const T *Tk = static_cast<const T *>(s.tr) + s.tr_off[lc * m.nsectors + s.sector[c]];
    T *mc = dm + s.mom_off[c] * nrhs;
    const T *mp = dm + s.mom_off[par] * nrhs;
    const int nq = m.ncomp * nrhs;
    if (m.transfer_kind == H2B_TRANSFER_DENSE) {
        // stored T is nin x nout (parent x child): op(T) = T^T (or T^H), column-contiguous in k
        A *Ms = sm, *Xs = sm + TG_M * TG_LD;
        for (int q0 = 0; q0 < nq; q0 += TG_Q) {
            const int nqc = min(TG_Q, nq - q0);
            for (int m0 = 0; m0 < nout; m0 += TG_M) {
                const int mt = min(TG_M, nout - m0);
                if constexpr (!MMA) {  // one right-hand side: FMA tile (an MMA would idle 7 of 8 columns)
                    A acc[TG_O];
                    tile_zero(acc);
                    tile_gemm(Tk, nin, true, conjt, m0, mt, nin, nqc,
                              [&](int kk, int q) -> A { return wide(mp[(int64_t)(q0 + q) * nin + kk]); }, Ms, Xs, acc);
#pragma unroll
                    for (int j = 0; j < TG_O; ++j) {
                        const int o = threadIdx.x + j * blockDim.x;
                        if (o < mt * nqc) {
                            T *dst = &mc[(int64_t)(q0 + o / mt) * nout + m0 + o % mt];
                            narrow(acc0 ? wide(*dst) + acc[j] : acc[j], *dst);
                        }
                    }
                } else {
                MmaAcc<A> acc;  // FP64 tensor cores (256 threads: 8 warps x 8 rows)
                acc.zero();
                tile_gemm_mma_l(true, m0, mt, nin, nqc,
                                [&](int i, int kk) -> A { return wide(cj(Tk[kk + (int64_t)i * nin], conjt)); },
                                [&](int kk, int q) -> A { return wide(mp[(int64_t)(q0 + q) * nin + kk]); }, Ms, Xs, acc);
                mma_store(acc, mt, nqc, [&](int i, int q, A v) {
                    T *dst = &mc[(int64_t)(q0 + q) * nout + m0 + i];
                    narrow(acc0 ? wide(*dst) + v : v, *dst);
                });
                }
            }
        }
        return;
    }
    const int mx = sep_bound(s, lp);
    A *bufa = sm, *bufb = sm + mx;
    for (int q = 0; q < nq; ++q) {
        for (int e = threadIdx.x; e < nin; e += blockDim.x) bufa[e] = wide(mp[(int64_t)q * nin + e]);
        __syncthreads();
        separable_block(Tk, &s.shape[3 * lp], &s.shape[3 * lc], m.dim, false, conjt, bufa, bufb,
                        mc + (int64_t)q * nout, acc0);
    }
}

// ---------------------------------------------------------------------------------------------
// C2: y[values] = alpha * sum_c op(C_c)^T l_c + beta * y[values]  (beta == 0 overwrites)
// ---------------------------------------------------------------------------------------------
template <class T, class V, bool MMA>
__global__ void __launch_bounds__(256)
leaf_disaggregate_kernel(DMap m, DSide s, const int *__restrict__ leaves, bool conjc, int nrhs,
                         const T *__restrict__ dm, V alpha, V beta, bool beta_zero, V *__restrict__ y,
                         int64_t ldy) {
    using A = typename ScalarTraits<T>::Acc;  // == V
    extern __shared__ unsigned char smem_raw[];
    A *Ms = reinterpret_cast<A *>(smem_raw), *Xs = Ms + TG_M * TG_LD;
    const int leaf = leaves[blockIdx.x];
    const int nc = ncoef_of(s, s.level[leaf]);
    const int v0 = s.value_ptr[leaf], nv = s.value_ptr[leaf + 1] - v0;
    const T *C = static_cast<const T *>(s.coll) + s.coll_off[leaf];
    const T *mom = dm + s.mom_off[leaf] * nrhs;
    for (int q0 = 0; q0 < nrhs; q0 += TG_Q) {
        const int nq = min(TG_Q, nrhs - q0);
        for (int m0 = 0; m0 < nv; m0 += TG_M) {
            const int mt = min(TG_M, nv - m0);
            if constexpr (!MMA) {  // one right-hand side: FMA tile
                A acc[TG_O];
                tile_zero(acc);
                for (int c = 0; c < m.ncomp; ++c)
                    tile_gemm(C + (int64_t)c * nc * nv, nc, true, conjc, m0, mt, nc, nq,
                              [&](int k, int q) -> A { return wide(mom[((int64_t)c * nrhs + q0 + q) * nc + k]); },
                              Ms, Xs, acc);
#pragma unroll
                for (int j = 0; j < TG_O; ++j) {
                    const int o = threadIdx.x + j * blockDim.x;
                    if (o < mt * nq) {
                        V *dst = &y[(int64_t)(q0 + o / mt) * ldy + s.value[v0 + m0 + o % mt]];
                        const V v = alpha * acc[j];
                        *dst = beta_zero ? v : v + beta * *dst;
                    }
                }
            } else {
            MmaAcc<A> acc;  // FP64 tensor cores (256 threads: 8 warps x 8 rows)
            acc.zero();
            for (int c = 0; c < m.ncomp; ++c) {
                const T *Cc = C + (int64_t)c * nc * nv;
                tile_gemm_mma_l(true, m0, mt, nc, nq,
                                [&](int i, int k) -> A { return wide(cj(Cc[k + (int64_t)i * nc], conjc)); },
                                [&](int k, int q) -> A { return wide(mom[((int64_t)c * nrhs + q0 + q) * nc + k]); },
                                Ms, Xs, acc);
            }
            mma_store(acc, mt, nq, [&](int i, int q, A v) {
                V *dst = &y[(int64_t)(q0 + q) * ldy + s.value[v0 + m0 + i]];
                const V w = alpha * v;
                *dst = beta_zero ? w : w + beta * *dst;
            });
            }
        }
    }
}

template <class V>
__global__ void zero_columns_kernel(int nrhs, int64_t n, V *y, int64_t ldy) {
    const int64_t total = n * nrhs;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x)
        y[(e / n) * ldy + (e % n)] = V{};
}

int block_for(int n, int lo = 32, int hi = 256) {
    int b = ((n + 31) / 32) * 32;
    return std::min(std::max(b, lo), hi);
}

template <class K>
cudaError_t allow_smem(K kernel, size_t bytes) {
    if (bytes > 48 * 1024)
        return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    return cudaSuccess;
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------------------------
#define H2B_DISPATCH_T(cplx, precision, ...)                                      \
    do {                                                                          \
        if (!(cplx) && (precision) == H2B_FP64) { using T = double; __VA_ARGS__; } \
        else if (!(cplx)) { using T = float; __VA_ARGS__; }                        \
        else if ((precision) == H2B_FP64) { using T = cdouble; __VA_ARGS__; }      \
        else { using T = cfloat; __VA_ARGS__; }                                    \
    } while (0)
#define H2B_DISPATCH_REAL(precision, ...)                                          \
    do {                                                                          \
        if ((precision) == H2B_FP64) { using T = double; __VA_ARGS__; }            \
        else { using T = float; __VA_ARGS__; }                                     \
    } while (0)
#define H2B_DISPATCH_CPLX(precision, ...)                                          \
    do {                                                                          \
        if ((precision) == H2B_FP64) { using T = cdouble; __VA_ARGS__; }           \
        else { using T = cfloat; __VA_ARGS__; }                                    \
    } while (0)

cudaError_t launch_leaf_aggregate(bool cplx, int precision, const DMap &m, const DSide &s,
                                  const int *leaves, int nleaves, int maxcoef, bool conjc,
                                  const FarArgs &fa, const void *x, int64_t ldx, cudaStream_t st) {
    if (nleaves == 0) return cudaSuccess;
    cudaError_t err = cudaSuccess;
    if (!cplx) {
        H2B_DISPATCH_REAL(precision, {
            if (fa.nrhs >= 2 && fa.nrhs <= 16 && maxcoef <= 64) {
                leaf_aggregate_warp_kernel<T><<<(nleaves + 7) / 8, 256, 0, st>>>(
                    m, s, leaves, nleaves, fa.nrhs, static_cast<const double *>(x), ldx, static_cast<T *>(fa.am));
                break;
            }
            auto kern = fa.nrhs > 1 ? &leaf_aggregate_kernel<T, double, true> : &leaf_aggregate_kernel<T, double, false>;
            err = allow_smem(kern, tile_smem<double>());
            if (err == cudaSuccess)
                kern<<<nleaves, 256, tile_smem<double>(), st>>>(
                    m, s, leaves, conjc, fa.nrhs, static_cast<const double *>(x), ldx, static_cast<T *>(fa.am));
        });
    } else {
        H2B_DISPATCH_CPLX(precision, {
            auto kern = fa.nrhs > 1 ? &leaf_aggregate_kernel<T, cdouble, true> : &leaf_aggregate_kernel<T, cdouble, false>;
            err = allow_smem(kern, tile_smem<cdouble>());
            if (err == cudaSuccess)
                kern<<<nleaves, 256, tile_smem<cdouble>(), st>>>(
                    m, s, leaves, conjc, fa.nrhs, static_cast<const cdouble *>(x), ldx, static_cast<T *>(fa.am));
        });
    }
    return err != cudaSuccess ? err : cudaGetLastError();
}

cudaError_t launch_transfer_up(bool cplx, int precision, const DMap &m, const DSide &s,
                               const int *nodes, int nnodes, bool conjt, const FarArgs &fa,
                               int maxcoef, int maxsep, cudaStream_t st) {
    if (nnodes == 0) return cudaSuccess;
    // real maps, dense transfers of at most 64 coefficients, 2-16 right-hand sides: a warp per child
    const int nqw = m.ncomp * fa.nrhs;
    if (!cplx && m.transfer_kind == H2B_TRANSFER_DENSE && nqw >= 2 && nqw <= 16 && maxcoef <= 64 && m.nsectors <= 8) {
        cudaError_t e = precision == H2B_FP64 ? warp_transfer_up<double>(m, s, nodes, nnodes, fa.nrhs, fa.am, st)
                                              : warp_transfer_up<float>(m, s, nodes, nnodes, fa.nrhs, fa.am, st);
        return e != cudaSuccess ? e : cudaGetLastError();
    }
    const int bs = m.transfer_kind == H2B_TRANSFER_DENSE ? 256 : block_for(maxcoef);
    cudaError_t err = cudaSuccess;
    if (m.transfer_kind == H2B_TRANSFER_SEPARABLE) {
        H2B_DISPATCH_T(cplx, precision, {
            err = launch_transfer_sep<T, true>(m, s, nodes, nnodes, nullptr, conjt, fa.nrhs, fa.am, maxsep, st);
        });
        return err;
    }
    H2B_DISPATCH_T(cplx, precision, {
        using A = typename ScalarTraits<T>::Acc;
        const size_t sm = m.transfer_kind == H2B_TRANSFER_DENSE ? tile_smem<A>()
                                                                 : 3 * (size_t)maxsep * sizeof(A);
        const int nq = m.ncomp * fa.nrhs;
        auto kern = nq > 1 ? &transfer_up_kernel<T, true> : &transfer_up_kernel<T, false>;
        err = allow_smem(kern, sm);
        if (err == cudaSuccess)
            kern<<<nnodes, bs, sm, st>>>(m, s, nodes, conjt, fa.nrhs, static_cast<T *>(fa.am));
    });
    return err != cudaSuccess ? err : cudaGetLastError();
}

namespace {
int fft_groups(int maxt, size_t scalar) {
    int g = 4;
    while (g > 1 && (size_t)g * (maxt + 3 * FFT_NMAX) * scalar > 200 * 1024) --g;
    return g;
}
}  // namespace

// the pruned real-map transforms (complex maps keep the general ones)
template <class T>
cudaError_t launch_pruned_in(const DSide &s, const int *nodes, int ntrans, bool inverse, int nq,
                             const FarArgs &fa, cudaStream_t st) {
    if constexpr (ScalarTraits<T>::is_complex) {
        return cudaErrorInvalidValue;
    } else {
        using S = typename ScalarTraits<T>::Complex;
        toeplitz_in_cube4_real_kernel<T><<<(ntrans + PR_G - 1) / PR_G, PR_T * PR_G, 0, st>>>(
            s, nodes, ntrans, inverse, nq, fa.nrhs, static_cast<const T *>(fa.am), static_cast<S *>(fa.as));
        return cudaGetLastError();
    }
}

template <class T>
cudaError_t launch_pruned_out(const DSide &s, const int *nodes, int ntrans, bool inverse, int nq,
                              const FarArgs &fa, cudaStream_t st) {
    if constexpr (ScalarTraits<T>::is_complex) {
        return cudaErrorInvalidValue;
    } else {
        using S = typename ScalarTraits<T>::Complex;
        toeplitz_out_cube4_real_kernel<T><<<(ntrans + PR_G - 1) / PR_G, PR_T * PR_G, 0, st>>>(
            s, nodes, ntrans, inverse, nq, fa.nrhs, static_cast<const S *>(fa.ds), static_cast<T *>(fa.dm));
        return cudaGetLastError();
    }
}

cudaError_t launch_toeplitz_in(bool cplx, int precision, const DMap &m, const DSide &s,
                               const int *nodes, int nnodes, bool inverse, const FarArgs &fa,
                               int maxtsize, int maxaxis, cudaStream_t st) {
    if (nnodes == 0) return cudaSuccess;
    const bool cube7 = m.cube_ts == 7;
    cudaError_t err = cudaSuccess;
    H2B_DISPATCH_T(cplx, precision, {
        using S = typename ScalarTraits<T>::Complex;
        const int G = fft_groups(maxtsize, sizeof(cdouble));
        const size_t sm = (size_t)G * (maxtsize + 3 * FFT_NMAX) * sizeof(cdouble);
        const int ntrans = nnodes * m.ncomp * fa.nrhs;
        auto launch = [&](auto kern) {
            cudaError_t e2 = allow_smem(kern, sm);
            if (e2 == cudaSuccess)
                e2 = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                          cudaSharedmemCarveoutMaxShared);
            if (e2 == cudaSuccess)
                kern<<<(ntrans + G - 1) / G, G * FFT_T, sm, st>>>(
                    m, s, nodes, ntrans, inverse, fa.nrhs, maxtsize, static_cast<const T *>(fa.am), static_cast<S *>(fa.as));
            return e2;
        };
        if (!cplx && cube7 && m.half_spectrum) {
            err = launch_pruned_in<T>(s, nodes, ntrans, inverse, m.ncomp * fa.nrhs, fa, st);
            break;
        }
        err = cube7 ? launch(toeplitz_in_kernel<T, 7, 7>)
                    : (maxaxis <= 7 ? launch(toeplitz_in_kernel<T, 7, 0>) : launch(toeplitz_in_kernel<T, 15, 0>));
    });
    return err != cudaSuccess ? err : cudaGetLastError();
}

bool i2o_grouped_eligible(bool cplx, int precision, const DMap &m, int nq, int maxcoef) {
    if (m.coupling_kind != H2B_COUPLING_DENSE || (cplx ? 2 : 1) * nq > GT_MAX_COLS) return false;
    // the chunk's sums (FP64) and two stages of the block piece and the moments (storage type)
    // fit in a CTA's shared memory
    const size_t a = cplx ? sizeof(cdouble) : sizeof(double);
    const size_t e = (cplx ? 2 : 1) * (precision == H2B_FP32 ? 4 : 8);
    const size_t nb = cplx ? gt_nb<cdouble>() : gt_nb<double>();
    return 2 * (TG_M * TG_LD + nb * TG_K * TG_Q) * e + (size_t)GT_R * nq * maxcoef * a <= 227u * 1024u - 4096u;
}

cudaError_t launch_i2o_grouped(bool cplx, int precision, const DMap &m, const DSide &recv, const DSide &src,
                               const GroupTiles &gt, int maxcoef, const FarArgs &fa, cudaStream_t st) {
    if (gt.nchunks == 0) return cudaSuccess;
    const int nq = m.ncomp * fa.nrhs;
    cudaError_t err = cudaSuccess;
    H2B_DISPATCH_T(cplx, precision, {
        using A = typename ScalarTraits<T>::Acc;
        const size_t sm = (size_t)GT_R * nq * maxcoef * sizeof(A) +
                          2 * (size_t)(TG_M * TG_LD + gt_nb<A>() * TG_K * TG_Q) * sizeof(T);
        auto kern = &i2o_grouped_kernel<T>;
        err = allow_smem(kern, sm);
        if (err == cudaSuccess)
            kern<<<gt.nchunks, 256, sm, st>>>(m, recv, src, gt, fa.mode, fa.nrhs, maxcoef,
                                              static_cast<const T *>(fa.am), static_cast<T *>(fa.dm));
    });
    return err != cudaSuccess ? err : cudaGetLastError();
}

cudaError_t launch_toeplitz_out(bool cplx, int precision, const DMap &m, const DSide &s,
                                const int *nodes, int nnodes, bool inverse, const FarArgs &fa,
                                int maxtsize, int maxaxis, cudaStream_t st) {
    if (nnodes == 0) return cudaSuccess;
    const bool cube7 = m.cube_ts == 7;
    cudaError_t err = cudaSuccess;
    H2B_DISPATCH_T(cplx, precision, {
        using S = typename ScalarTraits<T>::Complex;
        const int G = fft_groups(maxtsize, sizeof(cdouble));
        const size_t sm = (size_t)G * (maxtsize + 3 * FFT_NMAX) * sizeof(cdouble);
        const int ntrans = nnodes * m.ncomp * fa.nrhs;
        auto launch = [&](auto kern) {
            cudaError_t e2 = allow_smem(kern, sm);
            if (e2 == cudaSuccess)
                e2 = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                          cudaSharedmemCarveoutMaxShared);
            if (e2 == cudaSuccess)
                kern<<<(ntrans + G - 1) / G, G * FFT_T, sm, st>>>(
                    m, s, nodes, ntrans, inverse, fa.nrhs, maxtsize, static_cast<const S *>(fa.ds), static_cast<T *>(fa.dm));
            return e2;
        };
        if (!cplx && cube7 && m.half_spectrum) {
            err = launch_pruned_out<T>(s, nodes, ntrans, inverse, m.ncomp * fa.nrhs, fa, st);
            break;
        }
        err = cube7 ? launch(toeplitz_out_kernel<T, 7, 7>)
                    : (maxaxis <= 7 ? launch(toeplitz_out_kernel<T, 7, 0>) : launch(toeplitz_out_kernel<T, 15, 0>));
    });
    return err != cudaSuccess ? err : cudaGetLastError();
}

cudaError_t launch_i2o(bool cplx, int precision, const DMap &m, const DSide &recv,
                       const DSide &src, const int *nodes, int nnodes, const FarArgs &fa,
                       int maxcoef, int maxtsize, int maxhalf, cudaStream_t st) {
    if (nnodes == 0) return cudaSuccess;
    if (i2o_umma_eligible(cplx, precision, m, m.ncomp * fa.nrhs))
        return launch_i2o_umma(cplx, m, recv, src, nodes, nnodes, fa, maxcoef, st);
    // Toeplitz: one thread per stored frequency (half spectra hold (n1/2 + 1) * n2 * n3 of them);
    // dense: the tile product's 256 threads
    const bool toep = m.coupling_kind == H2B_COUPLING_TOEPLITZ;
    const bool diag = m.coupling_kind == H2B_COUPLING_DIAGONAL;
    const int bs = toep ? block_for(m.half_spectrum ? maxhalf : maxtsize, 32, 512)
                        : (diag ? block_for(maxcoef, 64, 256) : 256);
    cudaError_t err = cudaSuccess;
    H2B_DISPATCH_T(cplx, precision, {
        using S = typename ScalarTraits<T>::Complex;
        const size_t sm = (toep || diag) ? 0 : tile_smem<typename ScalarTraits<T>::Acc>();
        auto kern = m.ncomp * fa.nrhs > 1 ? &i2o_kernel<T, true> : &i2o_kernel<T, false>;
        err = allow_smem(kern, sm);
        if (err == cudaSuccess)
            kern<<<nnodes, bs, sm, st>>>(m, recv, src, nodes, fa.mode, fa.nrhs,
                                                  static_cast<const T *>(fa.am), static_cast<T *>(fa.dm),
                                                  static_cast<const S *>(fa.as), static_cast<S *>(fa.ds));
    });
    return err != cudaSuccess ? err : cudaGetLastError();
}

cudaError_t launch_i2o_siblings(bool cplx, int precision, const DMap &m, const DSide &recv,
                                const SibGroups &g, int maxslen, const FarArgs &fa, cudaStream_t st) {
    if (g.ngroups == 0) return cudaSuccess;
    const int nq = m.ncomp * fa.nrhs;
    const int bs = block_for(maxslen, 32, 512);
    H2B_DISPATCH_T(cplx, precision, {
        using S = typename ScalarTraits<T>::Complex;
        // several right-hand sides per CTA share each kernel value load (one-wide blocks reload
        // them per right-hand side, which costs more than the lower occupancy of the wider block):
        // four with FP32 accumulators, two with FP64 ones (four would spill)
        constexpr bool f32 = sizeof(typename ScalarTraits<T>::Real) == 4;
        constexpr int QB = f32 ? 4 : 2;
        // one right-hand side: the (slot, frequency) form (2 % faster on the benchmark map);
        // blocks of right-hand sides: the frequency-per-thread form, which reuses each source
        // value from registers for the 8 slots (7 % faster than the slot form at 16)
        if (nq == 1)
            i2o_slot_kernel<T, 1, 4><<<dim3(g.ngroups, (maxslen + 31) / 32, 1), 256, 0, st>>>(
                m, recv, g, fa.mode, fa.nrhs, static_cast<const S *>(fa.as), static_cast<S *>(fa.ds));
        else if (!f32 && nq >= 8) {
            // FP64 spectra, blocks of 8+ right-hand sides: the FP64 tensor-core form, one warp per
            // frequency (16 RHS on the benchmark map: 3.64 vs 3.79 ms per product). FP32 spectra keep
            // the FMA form below: on the tensor pipe, shared with the near field's products, the
            // served step measured 3.32 ms against 2.54.
            i2o_sibling_dmma_kernel<S, 2><<<dim3(g.ngroups, (maxslen + 7) / 8, (nq + 15) / 16), 256, 0, st>>>(
                m, recv, g, fa.mode, fa.nrhs, static_cast<const S *>(fa.as), static_cast<S *>(fa.ds));
        } else if (f32 && maxslen <= 256) {
            // FP32: two threads per frequency, 4 slots x 8 right-hand sides each (3 % faster than
            // 8 slots x 4 on the benchmark map; unrolling entries or 2-wide blocks were slower)
            const int et = block_for(maxslen, 32, 256);
            i2o_sibling_kernel<T, 8, 4, 1><<<dim3(g.ngroups, (nq + 7) / 8), 2 * et, 0, st>>>(
                m, recv, g, fa.mode, fa.nrhs, et, static_cast<const S *>(fa.as), static_cast<S *>(fa.ds));
        } else {
            i2o_sibling_kernel<T, QB, 8, 1><<<dim3(g.ngroups, (nq + QB - 1) / QB), bs, 0, st>>>(
                m, recv, g, fa.mode, fa.nrhs, bs, static_cast<const S *>(fa.as), static_cast<S *>(fa.ds));
        }
    });
    return cudaGetLastError();
}

cudaError_t launch_transfer_down(bool cplx, int precision, const DMap &m, const DSide &s,
                                 const int *nodes, int nnodes, const uint8_t *received,
                                 const FarArgs &fa, int maxcoef, int maxsep, cudaStream_t st) {
    if (nnodes == 0) return cudaSuccess;
    const int nqw = m.ncomp * fa.nrhs;
    if (!cplx && m.transfer_kind == H2B_TRANSFER_DENSE && nqw >= 2 && nqw <= 16 && maxcoef <= 64) {
        if (precision == H2B_FP64) warp_transfer_down<double>(m, s, nodes, nnodes, received, fa.nrhs, fa.dm, st);
        else warp_transfer_down<float>(m, s, nodes, nnodes, received, fa.nrhs, fa.dm, st);
        return cudaGetLastError();
    }
    const int bs = m.transfer_kind == H2B_TRANSFER_DENSE ? 256 : block_for(maxcoef, 64, 256);
    const bool conjt = fa.mode == H2B_ADJOINT;
    cudaError_t err = cudaSuccess;
    if (m.transfer_kind == H2B_TRANSFER_SEPARABLE) {
        H2B_DISPATCH_T(cplx, precision, {
            err = launch_transfer_sep<T, false>(m, s, nodes, nnodes, received, conjt, fa.nrhs, fa.dm, maxsep, st);
        });
        return err;
    }
    H2B_DISPATCH_T(cplx, precision, {
        using A = typename ScalarTraits<T>::Acc;
        const size_t sm = m.transfer_kind == H2B_TRANSFER_DENSE ? tile_smem<A>()
                                                                 : 2 * (size_t)maxsep * sizeof(A);
        const int nq = m.ncomp * fa.nrhs;
        auto kern = nq > 1 ? &transfer_down_kernel<T, true> : &transfer_down_kernel<T, false>;
        err = allow_smem(kern, sm);
        if (err == cudaSuccess)
            kern<<<nnodes, bs, sm, st>>>(m, s, nodes, received, conjt, fa.nrhs,
                                                           static_cast<T *>(fa.dm));
    });
    return err != cudaSuccess ? err : cudaGetLastError();
}

cudaError_t launch_leaf_disaggregate(bool cplx, int precision, const DMap &m, const DSide &s,
                                     const int *leaves, int nleaves, bool conjc, const FarArgs &fa,
                                     cdouble alpha, cdouble beta, void *y, int64_t ldy,
                                     cudaStream_t st) {
    if (nleaves == 0) return cudaSuccess;
    const int bs = 256;
    cudaError_t err = cudaSuccess;
    if (!cplx) {
        const bool bz = beta.x == 0.0;
        H2B_DISPATCH_REAL(precision, {
            if (fa.nrhs >= 2 && fa.nrhs <= 16) {  // a warp per leaf
                leaf_disaggregate_warp_kernel<T><<<(nleaves + 7) / 8, 256, 0, st>>>(
                    m, s, leaves, nleaves, fa.nrhs, static_cast<const T *>(fa.dm), alpha.x, beta.x, bz,
                    static_cast<double *>(y), ldy);
                break;
            }
            auto kern = fa.nrhs > 1 ? &leaf_disaggregate_kernel<T, double, true> : &leaf_disaggregate_kernel<T, double, false>;
            err = allow_smem(kern, tile_smem<double>());
            if (err == cudaSuccess)
                kern<<<nleaves, bs, tile_smem<double>(), st>>>(
                    m, s, leaves, conjc, fa.nrhs, static_cast<const T *>(fa.dm), alpha.x, beta.x, bz,
                    static_cast<double *>(y), ldy);
        });
    } else {
        const bool bz = beta.x == 0.0 && beta.y == 0.0;
        H2B_DISPATCH_CPLX(precision, {
            auto kern = fa.nrhs > 1 ? &leaf_disaggregate_kernel<T, cdouble, true> : &leaf_disaggregate_kernel<T, cdouble, false>;
            err = allow_smem(kern, tile_smem<cdouble>());
            if (err == cudaSuccess)
                kern<<<nleaves, bs, tile_smem<cdouble>(), st>>>(
                    m, s, leaves, conjc, fa.nrhs, static_cast<const T *>(fa.dm), alpha, beta, bz,
                    static_cast<cdouble *>(y), ldy);
        });
    }
    return err != cudaSuccess ? err : cudaGetLastError();
}

cudaError_t launch_zero_columns(bool cplx, int nrhs, int64_t n, void *y, int64_t ldy, cudaStream_t st) {
    if (n == 0 || nrhs == 0) return cudaSuccess;
    const int64_t total = n * nrhs;
    const int grid = (int)std::min<int64_t>((total + 255) / 256, 148 * 8);
    if (cplx)
        zero_columns_kernel<cdouble><<<grid, 256, 0, st>>>(nrhs, n, static_cast<cdouble *>(y), ldy);
    else
        zero_columns_kernel<double><<<grid, 256, 0, st>>>(nrhs, n, static_cast<double *>(y), ldy);
    return cudaGetLastError();
}

}  // namespace h2b
