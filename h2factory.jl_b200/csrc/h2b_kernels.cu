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

#include "h2b_internal.cuh"

namespace h2b {

namespace {

constexpr int RCH = 4;   // right-hand sides per register chunk
constexpr int JT = 64;   // x values staged in shared memory per tile

__device__ __forceinline__ int ncoef_of(const DSide &s, int lvl) {
    return s.shape[3 * lvl] * s.shape[3 * lvl + 1] * s.shape[3 * lvl + 2];
}

// Bound on every intermediate of a separable contraction between levels lp and lp + 1.
__device__ __forceinline__ int sep_bound(const DSide &s, int lp) {
    int b = 1;
    for (int d = 0; d < 3; ++d) b *= max(s.shape[3 * lp + d], s.shape[3 * (lp + 1) + d]);
    return b;
}

__device__ __forceinline__ double shfl_x(double v, int o) { return __shfl_xor_sync(0xffffffffu, v, o); }
__device__ __forceinline__ float shfl_x(float v, int o) { return __shfl_xor_sync(0xffffffffu, v, o); }
template <class R> __device__ __forceinline__ Cx<R> shfl_x(Cx<R> v, int o) {
    return {shfl_x(v.x, o), shfl_x(v.y, o)};
}
template <class T> __device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += shfl_x(v, o);
    return v;
}

// ---------------------------------------------------------------------------------------------
// A1: m_leaf[c][r] = op(C_c) x[values]   (op = conj for adjoint maps with conjugating leaves)
// ---------------------------------------------------------------------------------------------
template <class T, class V>
__global__ void leaf_aggregate_kernel(DMap m, DSide s, const int *__restrict__ leaves, bool conjc,
                                      int nrhs, const V *__restrict__ x, int64_t ldx,
                                      T *__restrict__ am) {
    __shared__ T xs[JT * RCH];
    const int leaf = leaves[blockIdx.x];
    const int nc = ncoef_of(s, s.level[leaf]);
    const int v0 = s.value_ptr[leaf], nv = s.value_ptr[leaf + 1] - v0;
    const T *C = static_cast<const T *>(s.coll) + s.coll_off[leaf];
    T *mom = am + s.mom_off[leaf] * nrhs;
    for (int c = 0; c < m.ncomp; ++c) {
        const T *Cc = C + (int64_t)c * nc * nv;
        for (int r0 = 0; r0 < nrhs; r0 += RCH) {
            const int rc = min(RCH, nrhs - r0);
            for (int a0 = 0; a0 < nc; a0 += blockDim.x) {
                const int a = a0 + threadIdx.x;
                T acc[RCH];
#pragma unroll
                for (int q = 0; q < RCH; ++q) acc[q] = sc_zero<T>();
                for (int j0 = 0; j0 < nv; j0 += JT) {
                    const int jt = min(JT, nv - j0);
                    __syncthreads();
                    for (int e = threadIdx.x; e < JT * RCH; e += blockDim.x) {
                        const int jj = e / RCH, q = e % RCH;
                        xs[e] = (jj < jt && q < rc)
                                    ? to_t(x[(int64_t)(r0 + q) * ldx + s.value[v0 + j0 + jj]], T{})
                                    : sc_zero<T>();
                    }
                    __syncthreads();
                    if (a < nc) {
                        const T *col = Cc + (int64_t)j0 * nc + a;
#pragma unroll 4
                        for (int jj = 0; jj < jt; ++jj) {
                            const T cij = cj(col[(int64_t)jj * nc], conjc);
#pragma unroll
                            for (int q = 0; q < RCH; ++q) acc[q] = acc[q] + cij * xs[jj * RCH + q];
                        }
                    }
                }
                if (a < nc)
                    for (int q = 0; q < rc; ++q) mom[((int64_t)c * nrhs + r0 + q) * nc + a] = acc[q];
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
template <class T>
__device__ void separable_block(const T *M, const int *sp, const int *sc, int dim, bool up, bool cjg,
                                T *a, T *b, T *out, bool accumulate) {
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
            T acc = sc_zero<T>();
            for (int k = 0; k < cur[ax]; ++k) {
                int src[3] = {idx[0], idx[1], idx[2]};
                src[ax] = k;
                // up: op(M)[row,k] = M[row + k*ld]; down: M^T[row,k] = M[k + row*ld]
                const T mk = up ? fac[ax][row + k * ld] : fac[ax][k + row * ld];
                acc = acc + cj(mk, cjg) * a[src[0] + cur[0] * (src[1] + cur[1] * src[2])];
            }
            b[e] = acc;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < total; e += blockDim.x) a[e] = b[e];
        __syncthreads();
        cur[0] = nxt[0]; cur[1] = nxt[1]; cur[2] = nxt[2];
    }
    const int total = fout[0] * fout[1] * fout[2];
    for (int e = threadIdx.x; e < total; e += blockDim.x) out[e] = accumulate ? out[e] + a[e] : a[e];
    __syncthreads();
}

// ---------------------------------------------------------------------------------------------
// A2: m_p = sum over children of op(T_{level(c), sector(c)}) m_c, first child overwriting.
// ---------------------------------------------------------------------------------------------
template <class T>
__global__ void transfer_up_kernel(DMap m, DSide s, const int *__restrict__ nodes, bool conjt,
                                   int nrhs, T *__restrict__ am) {
    extern __shared__ unsigned char smem_raw[];
    T *sm = reinterpret_cast<T *>(smem_raw);
    const int p = nodes[blockIdx.x];
    const int lp = s.level[p], lc = lp + 1;
    const int nout = ncoef_of(s, lp), nin = ncoef_of(s, lc);
    T *mp = am + s.mom_off[p] * nrhs;
    const int c0 = s.child_ptr[p], c1 = s.child_ptr[p + 1];
    const int nq = m.ncomp * nrhs;
    if (m.transfer_kind == H2B_TRANSFER_DENSE) {
        // children split over `ns` thread groups of `npad` threads, partial sums reduced in smem
        const int npad = ((nout + 31) / 32) * 32;
        const int ns = npad <= (int)blockDim.x ? (int)blockDim.x / npad : 1;
        const int sidx = threadIdx.x / npad;
        for (int q = 0; q < nq; ++q)
            for (int a0 = 0; a0 < nout; a0 += (ns > 1 ? npad : (int)blockDim.x)) {
                const int a = a0 + (ns > 1 ? (int)threadIdx.x % npad : (int)threadIdx.x);
                T acc = sc_zero<T>();
                if (sidx < ns && a < nout)
                    for (int k = c0 + sidx; k < c1; k += ns) {
                        const int ch = s.child[k];
                        const T *Tk = static_cast<const T *>(s.tr) + s.tr_off[lc * m.nsectors + s.sector[ch]];
                        const T *mc = am + s.mom_off[ch] * nrhs + (int64_t)q * nin;
#pragma unroll 4
                        for (int b = 0; b < nin; ++b) acc = acc + cj(Tk[a + (int64_t)b * nout], conjt) * mc[b];
                    }
                if (ns > 1) {
                    if (sidx < ns) sm[sidx * npad + (threadIdx.x % npad)] = acc;
                    __syncthreads();
                    if (threadIdx.x < npad && a0 + threadIdx.x < nout) {
                        T sum = sm[threadIdx.x];
                        for (int w = 1; w < ns; ++w) sum = sum + sm[w * npad + threadIdx.x];
                        mp[(int64_t)q * nout + a0 + threadIdx.x] = sum;
                    }
                    __syncthreads();
                } else if (a < nout) {
                    mp[(int64_t)q * nout + a] = acc;
                }
            }
        return;
    }
    const int mx = sep_bound(s, lp);
    T *bufa = sm, *bufb = sm + mx, *acc = sm + 2 * mx;
    for (int q = 0; q < nq; ++q) {
        for (int k = c0; k < c1; ++k) {
            const int ch = s.child[k];
            const T *Tk = static_cast<const T *>(s.tr) + s.tr_off[lc * m.nsectors + s.sector[ch]];
            const T *mc = am + s.mom_off[ch] * nrhs + (int64_t)q * nin;
            for (int e = threadIdx.x; e < nin; e += blockDim.x) bufa[e] = mc[e];
            __syncthreads();
            separable_block(Tk, &s.shape[3 * lp], &s.shape[3 * lc], m.dim, true, conjt, bufa, bufb,
                            acc, k != c0);
        }
        for (int e = threadIdx.x; e < nout; e += blockDim.x) mp[(int64_t)q * nout + e] = acc[e];
        __syncthreads();
    }
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

__device__ __forceinline__ TGeom tgeom(const DSide &s, int lvl, bool half) {
    TGeom g;
    for (int d = 0; d < 3; ++d) {
        g.sh[d] = s.shape[3 * lvl + d];
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
template <class T, int NMAX>
__global__ void __launch_bounds__(256) toeplitz_in_kernel(DMap m, DSide s, const int *__restrict__ nodes, int ntrans, bool inverse,
                                   int nrhs, int maxt, const T *__restrict__ am,
                                   typename ScalarTraits<T>::Complex *__restrict__ as) {
    using S = typename ScalarTraits<T>::Complex;
    using R = typename ScalarTraits<T>::Real;
    extern __shared__ unsigned char smem_raw[];
    const int grp = threadIdx.x / FFT_T, tl = threadIdx.x % FFT_T, ngrp = blockDim.x / FFT_T;
    S *a = reinterpret_cast<S *>(smem_raw) + (size_t)grp * (maxt + 3 * FFT_NMAX);
    S *tw = a + maxt;
    const int nq = m.ncomp * nrhs;
    const int t = blockIdx.x * ngrp + grp;
    const bool busy = t < ntrans;
    const int node = busy ? nodes[t / nq] : nodes[0];
    const int q = busy ? t % nq : 0;
    const TGeom g = tgeom(s, s.level[node], m.half_spectrum != 0);
    if (busy) {
        const T *mom = am + s.mom_off[node] * nrhs + (int64_t)q * g.nc;
        for (int e = tl; e < g.nt; e += FFT_T) {
            const int i1 = e % g.ts[0], i2 = (e / g.ts[0]) % g.ts[1], i3 = e / (g.ts[0] * g.ts[1]);
            S v = {(R)0, (R)0};
            if (i1 < g.sh[0] && i2 < g.sh[1] && i3 < g.sh[2])
                v = to_cx(mom[i1 + g.sh[0] * (i2 + g.sh[1] * i3)]);
            a[e] = v;
        }
    }
    dft_group<R, NMAX>(a, g, inverse, tw, tl, busy);
    if (busy) {
        S *spec = as + s.spec_off[node] * nrhs + (int64_t)q * g.slen;
        for (int e = tl; e < g.slen; e += FFT_T) {
            const int k1 = e % g.h0, r = e / g.h0;
            spec[e] = a[k1 + g.ts[0] * r];
        }
    }
}

// B3: moment(node) = corner(F^-1(spectrum(node)))   (overwrite)
template <class T, int NMAX>
__global__ void __launch_bounds__(256) toeplitz_out_kernel(DMap m, DSide s, const int *__restrict__ nodes, int ntrans, bool inverse,
                                    int nrhs, int maxt,
                                    const typename ScalarTraits<T>::Complex *__restrict__ ds,
                                    T *__restrict__ dm) {
    using S = typename ScalarTraits<T>::Complex;
    using R = typename ScalarTraits<T>::Real;
    extern __shared__ unsigned char smem_raw[];
    const int grp = threadIdx.x / FFT_T, tl = threadIdx.x % FFT_T, ngrp = blockDim.x / FFT_T;
    S *a = reinterpret_cast<S *>(smem_raw) + (size_t)grp * (maxt + 3 * FFT_NMAX);
    S *tw = a + maxt;
    const int nq = m.ncomp * nrhs;
    const int t = blockIdx.x * ngrp + grp;
    const bool busy = t < ntrans;
    const int node = busy ? nodes[t / nq] : nodes[0];
    const int q = busy ? t % nq : 0;
    const TGeom g = tgeom(s, s.level[node], m.half_spectrum != 0);
    if (busy) {
        const S *spec = ds + s.spec_off[node] * nrhs + (int64_t)q * g.slen;
        for (int e = tl; e < g.nt; e += FFT_T) {
            const int k1 = e % g.ts[0], r = e / g.ts[0];
            if (k1 < g.h0) {
                a[e] = spec[k1 + g.h0 * r];
            } else {
                const int k2 = r % g.ts[1], k3 = r / g.ts[1];
                const int m1 = g.ts[0] - k1, m2 = (g.ts[1] - k2) % g.ts[1], m3 = (g.ts[2] - k3) % g.ts[2];
                a[e] = conjg(spec[m1 + g.h0 * (m2 + g.ts[1] * m3)]);
            }
        }
    }
    dft_group<R, NMAX>(a, g, inverse, tw, tl, busy);
    if (busy) {
        T *mom = dm + s.mom_off[node] * nrhs + (int64_t)q * g.nc;
        for (int e = tl; e < g.nc; e += FFT_T) {
            const int i1 = e % g.sh[0], i2 = (e / g.sh[0]) % g.sh[1], i3 = e / (g.sh[0] * g.sh[1]);
            from_cx(a[i1 + g.ts[0] * (i2 + g.ts[1] * i3)], mom[e]);
        }
    }
}

// ---------------------------------------------------------------------------------------------
// B1/B2: l_r = sum over pairs of op(B_key) m_t (dense), d .* m_t (diagonal), or, for Toeplitz,
// S_r = sum K_key .* S_t on the spectra. op: identity / transpose / adjoint by map orientation
// (src/farinteractions/i2otranslations/i2oprotocol.jl:87-92, i2otranslationcollection.jl:367-495,
// toeplitzi2ocollection.jl:110-193). The first pair overwrites.
// ---------------------------------------------------------------------------------------------
template <class T>
__global__ void i2o_kernel(DMap m, DSide r, DSide t, const int *__restrict__ nodes, int mode,
                           int nrhs, const T *__restrict__ am, T *__restrict__ dm,
                           const typename ScalarTraits<T>::Complex *__restrict__ as,
                           typename ScalarTraits<T>::Complex *__restrict__ ds) {
    using S = typename ScalarTraits<T>::Complex;
    const int node = nodes[blockIdx.x];
    const int p0 = r.i2o_ptr[node], p1 = r.i2o_ptr[node + 1];
    const int lvl = r.level[node];
    const int nc = ncoef_of(r, lvl);
    const int nq = m.ncomp * nrhs;
    const bool adj = (mode == H2B_ADJOINT);
    // r.pair_src[p]: the source's moment (or spectrum) offset per unit rhs; r.pair_cpl[p]: the
    // coupling's element offset -- one load each per pair, no chained index lookups
    if (m.coupling_kind == H2B_COUPLING_TOEPLITZ) {
        const int nt = tgeom(r, lvl, m.half_spectrum != 0).slen;
        S *out = ds + r.spec_off[node] * nrhs;
        const S *K0 = static_cast<const S *>(m.cpl);
        for (int q = 0; q < nq; ++q)
            for (int e = threadIdx.x; e < nt; e += blockDim.x) {
                S acc = {0, 0};
                int p = p0;
                for (; p + 4 <= p1; p += 4) {
                    S kv[4], iv[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        kv[u] = K0[r.pair_cpl[p + u] + e];
                        iv[u] = as[r.pair_src[p + u] * nrhs + (int64_t)q * nt + e];
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) acc = acc + cj(kv[u], adj) * iv[u];
                }
                for (; p < p1; ++p)
                    acc = acc + cj(K0[r.pair_cpl[p] + e], adj) * as[r.pair_src[p] * nrhs + (int64_t)q * nt + e];
                out[(int64_t)q * nt + e] = acc;
            }
        return;
    }
    T *out = dm + r.mom_off[node] * nrhs;
    const T *B0 = static_cast<const T *>(m.cpl);
    if (m.coupling_kind == H2B_COUPLING_DIAGONAL) {
        for (int q = 0; q < nq; ++q)
            for (int a = threadIdx.x; a < nc; a += blockDim.x) {
                T acc = sc_zero<T>();
                for (int p = p0; p < p1; ++p) {
                    const T *D = B0 + r.pair_cpl[p];
                    acc = acc + cj(D[a], adj) * am[r.pair_src[p] * nrhs + (int64_t)q * nc + a];
                }
                out[(int64_t)q * nc + a] = acc;
            }
        return;
    }
    if (mode == H2B_FORWARD) {
        // thread per output row: B[a + b*nc] coalesced over a
        for (int q = 0; q < nq; ++q)
            for (int a = threadIdx.x; a < nc; a += blockDim.x) {
                T acc = sc_zero<T>();
                for (int p = p0; p < p1; ++p) {
                    const int snc = ncoef_of(t, t.level[r.i2o_src[p]]);
                    const T *B = B0 + r.pair_cpl[p];
                    const T *in = am + r.pair_src[p] * nrhs + (int64_t)q * snc;
                    for (int b = 0; b < snc; ++b) acc = acc + B[a + (int64_t)b * nc] * in[b];
                }
                out[(int64_t)q * nc + a] = acc;
            }
        return;
    }
    // transpose / adjoint: output a is column a of the stored block -> warp per output
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int q = 0; q < nq; ++q)
        for (int a = warp; a < nc; a += nw) {
            T acc = sc_zero<T>();
            for (int p = p0; p < p1; ++p) {
                const int snc = ncoef_of(t, t.level[r.i2o_src[p]]);
                const T *B = B0 + r.pair_cpl[p] + (int64_t)a * snc;
                const T *in = am + r.pair_src[p] * nrhs + (int64_t)q * snc;
                for (int b = lane; b < snc; b += 32) acc = acc + cj(B[b], adj) * in[b];
            }
            acc = warp_sum(acc);
            if (lane == 0) out[(int64_t)q * nc + a] = acc;
        }
}

// ---------------------------------------------------------------------------------------------
// C1: l_c = [l_c +] op(T_{level(c), sector(c)}) l_parent, op = transpose (adjoint for adjoint maps)
// ---------------------------------------------------------------------------------------------
template <class T>
__global__ void transfer_down_kernel(DMap m, DSide s, const int *__restrict__ nodes,
                                     const uint8_t *__restrict__ received, bool conjt, int nrhs,
                                     T *__restrict__ dm) {
    extern __shared__ unsigned char smem_raw[];
    T *sm = reinterpret_cast<T *>(smem_raw);
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
        // stored T is nin x nout (parent x child); output a reads column a: warp per output
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
        for (int q = 0; q < nq; ++q)
            for (int a = warp; a < nout; a += nw) {
                T acc = sc_zero<T>();
                const T *col = Tk + (int64_t)a * nin;
                const T *in = mp + (int64_t)q * nin;
                for (int b = lane; b < nin; b += 32) acc = acc + cj(col[b], conjt) * in[b];
                acc = warp_sum(acc);
                if (lane == 0) {
                    T *o = &mc[(int64_t)q * nout + a];
                    *o = acc0 ? *o + acc : acc;
                }
            }
        return;
    }
    const int mx = sep_bound(s, lp);
    T *bufa = sm, *bufb = sm + mx;
    for (int q = 0; q < nq; ++q) {
        for (int e = threadIdx.x; e < nin; e += blockDim.x) bufa[e] = mp[(int64_t)q * nin + e];
        __syncthreads();
        separable_block(Tk, &s.shape[3 * lp], &s.shape[3 * lc], m.dim, false, conjt, bufa, bufb,
                        mc + (int64_t)q * nout, acc0);
    }
}

// ---------------------------------------------------------------------------------------------
// C2: y[values] = alpha * sum_c op(C_c)^T l_c + beta * y[values]  (beta == 0 overwrites)
// ---------------------------------------------------------------------------------------------
template <class T, class V>
__global__ void leaf_disaggregate_kernel(DMap m, DSide s, const int *__restrict__ leaves, bool conjc,
                                         int nrhs, const T *__restrict__ dm, V alpha, V beta,
                                         bool beta_zero, V *__restrict__ y, int64_t ldy) {
    const int leaf = leaves[blockIdx.x];
    const int nc = ncoef_of(s, s.level[leaf]);
    const int v0 = s.value_ptr[leaf], nv = s.value_ptr[leaf + 1] - v0;
    const T *C = static_cast<const T *>(s.coll) + s.coll_off[leaf];
    const T *mom = dm + s.mom_off[leaf] * nrhs;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int j = warp; j < nv; j += nw) {
        for (int r = 0; r < nrhs; ++r) {
            T acc = sc_zero<T>();
            for (int c = 0; c < m.ncomp; ++c) {
                const T *col = C + (int64_t)c * nc * nv + (int64_t)j * nc;
                const T *l = mom + ((int64_t)c * nrhs + r) * nc;
                for (int a = lane; a < nc; a += 32) acc = acc + cj(col[a], conjc) * l[a];
            }
            acc = warp_sum(acc);
            if (lane == 0) {
                V *o = &y[(int64_t)r * ldy + s.value[v0 + j]];
                const V v = alpha * to_v(acc);
                *o = beta_zero ? v : v + beta * *o;
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
    const int bs = block_for(maxcoef, 64, 256);
    if (!cplx) {
        H2B_DISPATCH_REAL(precision,
            leaf_aggregate_kernel<T, double><<<nleaves, bs, 0, st>>>(
                m, s, leaves, conjc, fa.nrhs, static_cast<const double *>(x), ldx, static_cast<T *>(fa.am)));
    } else {
        H2B_DISPATCH_CPLX(precision,
            leaf_aggregate_kernel<T, cdouble><<<nleaves, bs, 0, st>>>(
                m, s, leaves, conjc, fa.nrhs, static_cast<const cdouble *>(x), ldx, static_cast<T *>(fa.am)));
    }
    return cudaGetLastError();
}

cudaError_t launch_transfer_up(bool cplx, int precision, const DMap &m, const DSide &s,
                               const int *nodes, int nnodes, bool conjt, const FarArgs &fa,
                               int maxcoef, int maxsep, cudaStream_t st) {
    if (nnodes == 0) return cudaSuccess;
    const int bs = m.transfer_kind == H2B_TRANSFER_DENSE ? 256 : block_for(maxcoef);
    cudaError_t err = cudaSuccess;
    H2B_DISPATCH_T(cplx, precision, {
        const size_t sm = m.transfer_kind == H2B_TRANSFER_DENSE ? (size_t)bs * sizeof(T)
                                                                 : 3 * (size_t)maxsep * sizeof(T);
        err = allow_smem(transfer_up_kernel<T>, sm);
        if (err == cudaSuccess)
            transfer_up_kernel<T><<<nnodes, bs, sm, st>>>(m, s, nodes, conjt, fa.nrhs, static_cast<T *>(fa.am));
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

cudaError_t launch_toeplitz_in(bool cplx, int precision, const DMap &m, const DSide &s,
                               const int *nodes, int nnodes, bool inverse, const FarArgs &fa,
                               int maxtsize, int maxaxis, cudaStream_t st) {
    if (nnodes == 0) return cudaSuccess;
    cudaError_t err = cudaSuccess;
    H2B_DISPATCH_T(cplx, precision, {
        using S = typename ScalarTraits<T>::Complex;
        const int G = fft_groups(maxtsize, sizeof(S));
        const size_t sm = (size_t)G * (maxtsize + 3 * FFT_NMAX) * sizeof(S);
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
        err = maxaxis <= 7 ? launch(toeplitz_in_kernel<T, 7>) : launch(toeplitz_in_kernel<T, 15>);
    });
    return err != cudaSuccess ? err : cudaGetLastError();
}

cudaError_t launch_toeplitz_out(bool cplx, int precision, const DMap &m, const DSide &s,
                                const int *nodes, int nnodes, bool inverse, const FarArgs &fa,
                                int maxtsize, int maxaxis, cudaStream_t st) {
    if (nnodes == 0) return cudaSuccess;
    cudaError_t err = cudaSuccess;
    H2B_DISPATCH_T(cplx, precision, {
        using S = typename ScalarTraits<T>::Complex;
        const int G = fft_groups(maxtsize, sizeof(S));
        const size_t sm = (size_t)G * (maxtsize + 3 * FFT_NMAX) * sizeof(S);
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
        err = maxaxis <= 7 ? launch(toeplitz_out_kernel<T, 7>) : launch(toeplitz_out_kernel<T, 15>);
    });
    return err != cudaSuccess ? err : cudaGetLastError();
}

cudaError_t launch_i2o(bool cplx, int precision, const DMap &m, const DSide &recv,
                       const DSide &src, const int *nodes, int nnodes, const FarArgs &fa,
                       int maxcoef, int maxtsize, int maxhalf, cudaStream_t st) {
    if (nnodes == 0) return cudaSuccess;
    // Toeplitz: one thread per stored frequency (half spectra hold (n1/2 + 1) * n2 * n3 of them)
    const int bs = m.coupling_kind == H2B_COUPLING_TOEPLITZ
                       ? block_for(m.half_spectrum ? maxhalf : maxtsize, 32, 512)
                       : block_for(maxcoef, 64, 256);
    H2B_DISPATCH_T(cplx, precision, {
        using S = typename ScalarTraits<T>::Complex;
        i2o_kernel<T><<<nnodes, bs, 0, st>>>(m, recv, src, nodes, fa.mode, fa.nrhs,
                                             static_cast<const T *>(fa.am), static_cast<T *>(fa.dm),
                                             static_cast<const S *>(fa.as), static_cast<S *>(fa.ds));
    });
    return cudaGetLastError();
}

cudaError_t launch_transfer_down(bool cplx, int precision, const DMap &m, const DSide &s,
                                 const int *nodes, int nnodes, const uint8_t *received,
                                 const FarArgs &fa, int maxcoef, int maxsep, cudaStream_t st) {
    if (nnodes == 0) return cudaSuccess;
    const int bs = block_for(maxcoef, 64, 256);
    const bool conjt = fa.mode == H2B_ADJOINT;
    cudaError_t err = cudaSuccess;
    H2B_DISPATCH_T(cplx, precision, {
        const size_t sm = m.transfer_kind == H2B_TRANSFER_DENSE ? 0 : 2 * (size_t)maxsep * sizeof(T);
        err = allow_smem(transfer_down_kernel<T>, sm);
        if (err == cudaSuccess)
            transfer_down_kernel<T><<<nnodes, bs, sm, st>>>(m, s, nodes, received, conjt, fa.nrhs,
                                                           static_cast<T *>(fa.dm));
    });
    return err != cudaSuccess ? err : cudaGetLastError();
}

cudaError_t launch_leaf_disaggregate(bool cplx, int precision, const DMap &m, const DSide &s,
                                     const int *leaves, int nleaves, bool conjc, const FarArgs &fa,
                                     cdouble alpha, cdouble beta, void *y, int64_t ldy,
                                     cudaStream_t st) {
    if (nleaves == 0) return cudaSuccess;
    const int bs = 128;
    if (!cplx) {
        const bool bz = beta.x == 0.0;
        H2B_DISPATCH_REAL(precision,
            leaf_disaggregate_kernel<T, double><<<nleaves, bs, 0, st>>>(
                m, s, leaves, conjc, fa.nrhs, static_cast<const T *>(fa.dm), alpha.x, beta.x, bz,
                static_cast<double *>(y), ldy));
    } else {
        const bool bz = beta.x == 0.0 && beta.y == 0.0;
        H2B_DISPATCH_CPLX(precision,
            leaf_disaggregate_kernel<T, cdouble><<<nleaves, bs, 0, st>>>(
                m, s, leaves, conjc, fa.nrhs, static_cast<const T *>(fa.dm), alpha, beta, bz,
                static_cast<cdouble *>(y), ldy));
    }
    return cudaGetLastError();
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
