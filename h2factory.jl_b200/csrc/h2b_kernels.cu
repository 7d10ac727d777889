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
//   near_*             D   nearmul!            src/nearinteractions/nearmul.jl:8-14
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
        for (int q = 0; q < nq; ++q)
            for (int a = threadIdx.x; a < nout; a += blockDim.x) {
                T acc = sc_zero<T>();
                for (int k = c0; k < c1; ++k) {
                    const int ch = s.child[k];
                    const T *Tk = static_cast<const T *>(s.tr) + s.tr_off[lc * m.nsectors + s.sector[ch]];
                    const T *mc = am + s.mom_off[ch] * nrhs + (int64_t)q * nin;
                    for (int b = 0; b < nin; ++b) acc = acc + cj(Tk[a + (int64_t)b * nout], conjt) * mc[b];
                }
                mp[(int64_t)q * nout + a] = acc;
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
// Multidimensional DFT of a column-major complex array in shared memory (AbstractFFTs
// conventions: forward e^{-2 pi i jk/n}; inverse e^{+2 pi i jk/n} and 1/n per axis).
// ---------------------------------------------------------------------------------------------
template <class R>
__device__ void dft_block(Cx<R> *&a, Cx<R> *&b, const int *ts, bool inverse, Cx<R> *tw) {
    const int total = ts[0] * ts[1] * ts[2];
    for (int ax = 0; ax < 3; ++ax) {
        const int n = ts[ax];
        if (n == 1) continue;
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            double sv, cv;
            sincospi(2.0 * k / n, &sv, &cv);
            tw[k] = {(R)cv, (R)(inverse ? sv : -sv)};
        }
        __syncthreads();
        const int stride = ax == 0 ? 1 : (ax == 1 ? ts[0] : ts[0] * ts[1]);
        const R scale = inverse ? (R)1 / (R)n : (R)1;
        for (int e = threadIdx.x; e < total; e += blockDim.x) {
            const int k = (e / stride) % n;
            const int base = e - k * stride;
            Cx<R> acc = {(R)0, (R)0};
            int w = 0;
            for (int j = 0; j < n; ++j) {
                acc = acc + a[base + j * stride] * tw[w];
                w += k;
                if (w >= n) w -= n;
            }
            b[e] = scale * acc;
        }
        __syncthreads();
        Cx<R> *t = a; a = b; b = t;
    }
}

// A3: spectrum(node) = F(pad(moment(node)))   (F = fft, or ifft for transpose maps)
template <class T>
__global__ void toeplitz_in_kernel(DMap m, DSide s, const int *__restrict__ nodes, bool inverse,
                                   int nrhs, const T *__restrict__ am,
                                   typename ScalarTraits<T>::Complex *__restrict__ as) {
    using S = typename ScalarTraits<T>::Complex;
    extern __shared__ unsigned char smem_raw[];
    const int node = nodes[blockIdx.x];
    const int lvl = s.level[node];
    const int *sh = &s.shape[3 * lvl];
    int ts[3] = {2 * sh[0] - 1, 2 * sh[1] - 1, 2 * sh[2] - 1};
    const int nt = ts[0] * ts[1] * ts[2], nc = sh[0] * sh[1] * sh[2];
    S *a = reinterpret_cast<S *>(smem_raw), *b = a + nt, *tw = b + nt;
    const T *mom = am + s.mom_off[node] * nrhs;
    S *spec = as + s.spec_off[node] * nrhs;
    for (int q = 0; q < m.ncomp * nrhs; ++q) {
        S *pa = a, *pb = b;
        for (int e = threadIdx.x; e < nt; e += blockDim.x) {
            const int i1 = e % ts[0], i2 = (e / ts[0]) % ts[1], i3 = e / (ts[0] * ts[1]);
            S v = {0, 0};
            if (i1 < sh[0] && i2 < sh[1] && i3 < sh[2])
                v = to_cx(mom[(int64_t)q * nc + i1 + sh[0] * (i2 + sh[1] * i3)]);
            pa[e] = v;
        }
        __syncthreads();
        dft_block(pa, pb, ts, inverse, tw);
        for (int e = threadIdx.x; e < nt; e += blockDim.x) spec[(int64_t)q * nt + e] = pa[e];
        __syncthreads();
    }
}

// B3: moment(node) = corner(F^-1(spectrum(node)))   (overwrite)
template <class T>
__global__ void toeplitz_out_kernel(DMap m, DSide s, const int *__restrict__ nodes, bool inverse,
                                    int nrhs, const typename ScalarTraits<T>::Complex *__restrict__ ds,
                                    T *__restrict__ dm) {
    using S = typename ScalarTraits<T>::Complex;
    extern __shared__ unsigned char smem_raw[];
    const int node = nodes[blockIdx.x];
    const int lvl = s.level[node];
    const int *sh = &s.shape[3 * lvl];
    int ts[3] = {2 * sh[0] - 1, 2 * sh[1] - 1, 2 * sh[2] - 1};
    const int nt = ts[0] * ts[1] * ts[2], nc = sh[0] * sh[1] * sh[2];
    S *a = reinterpret_cast<S *>(smem_raw), *b = a + nt, *tw = b + nt;
    T *mom = dm + s.mom_off[node] * nrhs;
    const S *spec = ds + s.spec_off[node] * nrhs;
    for (int q = 0; q < m.ncomp * nrhs; ++q) {
        S *pa = a, *pb = b;
        for (int e = threadIdx.x; e < nt; e += blockDim.x) pa[e] = spec[(int64_t)q * nt + e];
        __syncthreads();
        dft_block(pa, pb, ts, inverse, tw);
        for (int e = threadIdx.x; e < nc; e += blockDim.x) {
            const int i1 = e % sh[0], i2 = (e / sh[0]) % sh[1], i3 = e / (sh[0] * sh[1]);
            from_cx(pa[i1 + ts[0] * (i2 + ts[1] * i3)], mom[(int64_t)q * nc + e]);
        }
        __syncthreads();
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
    if (m.coupling_kind == H2B_COUPLING_TOEPLITZ) {
        const int *sh = &r.shape[3 * lvl];
        const int nt = (2 * sh[0] - 1) * (2 * sh[1] - 1) * (2 * sh[2] - 1);
        S *out = ds + r.spec_off[node] * nrhs;
        const S *K0 = static_cast<const S *>(m.cpl);
        for (int q = 0; q < nq; ++q)
            for (int e = threadIdx.x; e < nt; e += blockDim.x) {
                S acc = {0, 0};
                for (int p = p0; p < p1; ++p) {
                    const S *K = K0 + m.cpl_off[r.i2o_cpl[p]];
                    const S *in = as + t.spec_off[r.i2o_src[p]] * nrhs + (int64_t)q * nt;
                    acc = acc + cj(K[e], adj) * in[e];
                }
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
                    const int src = r.i2o_src[p];
                    const int snc = ncoef_of(t, t.level[src]);
                    const T *D = B0 + m.cpl_off[r.i2o_cpl[p]];
                    acc = acc + cj(D[a], adj) * am[t.mom_off[src] * nrhs + (int64_t)q * snc + a];
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
                    const int src = r.i2o_src[p];
                    const int snc = ncoef_of(t, t.level[src]);
                    const T *B = B0 + m.cpl_off[r.i2o_cpl[p]];
                    const T *in = am + t.mom_off[src] * nrhs + (int64_t)q * snc;
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
                const int src = r.i2o_src[p];
                const int snc = ncoef_of(t, t.level[src]);
                const T *B = B0 + m.cpl_off[r.i2o_cpl[p]] + (int64_t)a * snc;
                const T *in = am + t.mom_off[src] * nrhs + (int64_t)q * snc;
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

// ---------------------------------------------------------------------------------------------
// D: near field. Forward: block per test leaf, thread per row, B read column by column.
// Transposed: block per trial leaf, warp per output column of B, lanes along the column.
// ---------------------------------------------------------------------------------------------
template <class V>
__global__ void near_forward_kernel(DNear n, DSide rs, DSide cs, int nrhs, const V *__restrict__ x,
                                    int64_t ldx, V *__restrict__ y, int64_t ldy, V alpha, V beta,
                                    bool beta_zero) {
    __shared__ V xs[JT * RCH];
    const int g = blockIdx.x;
    const int row = n.row_leaf[g];
    const int r0v = rs.value_ptr[row], nr = rs.value_ptr[row + 1] - r0v;
    const int b0 = n.row_ptr[g], b1 = n.row_ptr[g + 1];
    const V *D = static_cast<const V *>(n.data);
    for (int r0 = 0; r0 < nrhs; r0 += RCH) {
        const int rc = min(RCH, nrhs - r0);
        for (int i0 = 0; i0 < nr; i0 += blockDim.x) {
            const int i = i0 + threadIdx.x;
            V acc[RCH];
#pragma unroll
            for (int q = 0; q < RCH; ++q) acc[q] = V{};
            for (int bb = b0; bb < b1; ++bb) {
                const int blk = n.row_blk[bb];
                const int col = n.blk_col[blk];
                const int c0v = cs.value_ptr[col], ncl = cs.value_ptr[col + 1] - c0v;
                const V *B = D + n.blk_off[blk];
                for (int j0 = 0; j0 < ncl; j0 += JT) {
                    const int jt = min(JT, ncl - j0);
                    __syncthreads();
                    for (int e = threadIdx.x; e < JT * RCH; e += blockDim.x) {
                        const int jj = e / RCH, q = e % RCH;
                        xs[e] = (jj < jt && q < rc) ? x[(int64_t)(r0 + q) * ldx + cs.value[c0v + j0 + jj]] : V{};
                    }
                    __syncthreads();
                    if (i < nr) {
                        const V *bc = B + (int64_t)j0 * nr + i;
#pragma unroll 8
                        for (int jj = 0; jj < jt; ++jj) {
                            const V bij = bc[(int64_t)jj * nr];
#pragma unroll
                            for (int q = 0; q < RCH; ++q) acc[q] = acc[q] + bij * xs[jj * RCH + q];
                        }
                    }
                }
            }
            if (i < nr)
                for (int q = 0; q < rc; ++q) {
                    V *o = &y[(int64_t)(r0 + q) * ldy + rs.value[r0v + i]];
                    const V v = alpha * acc[q];
                    *o = beta_zero ? v : v + beta * *o;
                }
        }
    }
}

template <class V>
__global__ void near_transposed_kernel(DNear n, DSide rs, DSide cs, bool adj, int nrhs,
                                       const V *__restrict__ x, int64_t ldx, V *__restrict__ y,
                                       int64_t ldy, V alpha, V beta, bool beta_zero) {
    extern __shared__ unsigned char smem_raw[];
    V *acc = reinterpret_cast<V *>(smem_raw);  // [ncl][RCH]
    const int g = blockIdx.x;
    const int col = n.col_leaf[g];
    const int c0v = cs.value_ptr[col], ncl = cs.value_ptr[col + 1] - c0v;
    const int b0 = n.col_ptr[g], b1 = n.col_ptr[g + 1];
    const V *D = static_cast<const V *>(n.data);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int r0 = 0; r0 < nrhs; r0 += RCH) {
        const int rc = min(RCH, nrhs - r0);
        for (int e = threadIdx.x; e < ncl * RCH; e += blockDim.x) acc[e] = V{};
        __syncthreads();
        for (int bb = b0; bb < b1; ++bb) {
            const int blk = n.col_blk[bb];
            const int row = n.blk_row[blk];
            const int r0v = rs.value_ptr[row], nr = rs.value_ptr[row + 1] - r0v;
            const V *B = D + n.blk_off[blk];
            for (int j = warp; j < ncl; j += nw) {
                const V *bc = B + (int64_t)j * nr;
                V part[RCH];
#pragma unroll
                for (int q = 0; q < RCH; ++q) part[q] = V{};
                for (int i = lane; i < nr; i += 32) {
                    const V bij = cj(bc[i], adj);
                    const int dof = rs.value[r0v + i];
#pragma unroll
                    for (int q = 0; q < RCH; ++q)
                        if (q < rc) part[q] = part[q] + bij * x[(int64_t)(r0 + q) * ldx + dof];
                }
#pragma unroll
                for (int q = 0; q < RCH; ++q) {
                    const V s = warp_sum(part[q]);
                    if (lane == 0) acc[j * RCH + q] = acc[j * RCH + q] + s;
                }
            }
        }
        __syncthreads();
        for (int e = threadIdx.x; e < ncl * rc; e += blockDim.x) {
            const int j = e / rc, q = e % rc;
            V *o = &y[(int64_t)(r0 + q) * ldy + cs.value[c0v + j]];
            const V v = alpha * acc[j * RCH + q];
            *o = beta_zero ? v : v + beta * *o;
        }
        __syncthreads();
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
    const int bs = block_for(maxcoef);
    cudaError_t err = cudaSuccess;
    H2B_DISPATCH_T(cplx, precision, {
        const size_t sm = m.transfer_kind == H2B_TRANSFER_DENSE ? 0 : 3 * (size_t)maxsep * sizeof(T);
        err = allow_smem(transfer_up_kernel<T>, sm);
        if (err == cudaSuccess)
            transfer_up_kernel<T><<<nnodes, bs, sm, st>>>(m, s, nodes, conjt, fa.nrhs, static_cast<T *>(fa.am));
    });
    return err != cudaSuccess ? err : cudaGetLastError();
}

cudaError_t launch_toeplitz_in(bool cplx, int precision, const DMap &m, const DSide &s,
                               const int *nodes, int nnodes, bool inverse, const FarArgs &fa,
                               int maxtsize, cudaStream_t st) {
    if (nnodes == 0) return cudaSuccess;
    const int bs = block_for(maxtsize, 64, 512);
    cudaError_t err = cudaSuccess;
    H2B_DISPATCH_T(cplx, precision, {
        using S = typename ScalarTraits<T>::Complex;
        const size_t sm = (2 * (size_t)maxtsize + 128) * sizeof(S);
        err = allow_smem(toeplitz_in_kernel<T>, sm);
        if (err == cudaSuccess)
            toeplitz_in_kernel<T><<<nnodes, bs, sm, st>>>(m, s, nodes, inverse, fa.nrhs,
                                                         static_cast<const T *>(fa.am), static_cast<S *>(fa.as));
    });
    return err != cudaSuccess ? err : cudaGetLastError();
}

cudaError_t launch_toeplitz_out(bool cplx, int precision, const DMap &m, const DSide &s,
                                const int *nodes, int nnodes, bool inverse, const FarArgs &fa,
                                int maxtsize, cudaStream_t st) {
    if (nnodes == 0) return cudaSuccess;
    const int bs = block_for(maxtsize, 64, 512);
    cudaError_t err = cudaSuccess;
    H2B_DISPATCH_T(cplx, precision, {
        using S = typename ScalarTraits<T>::Complex;
        const size_t sm = (2 * (size_t)maxtsize + 128) * sizeof(S);
        err = allow_smem(toeplitz_out_kernel<T>, sm);
        if (err == cudaSuccess)
            toeplitz_out_kernel<T><<<nnodes, bs, sm, st>>>(m, s, nodes, inverse, fa.nrhs,
                                                          static_cast<const S *>(fa.ds), static_cast<T *>(fa.dm));
    });
    return err != cudaSuccess ? err : cudaGetLastError();
}

cudaError_t launch_i2o(bool cplx, int precision, const DMap &m, const DSide &recv,
                       const DSide &src, const int *nodes, int nnodes, const FarArgs &fa,
                       int maxcoef, int maxtsize, cudaStream_t st) {
    if (nnodes == 0) return cudaSuccess;
    const int bs = m.coupling_kind == H2B_COUPLING_TOEPLITZ ? block_for(maxtsize, 64, 512)
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

cudaError_t launch_near(bool cplx, int mode, const DNear &n, const DSide &rows, const DSide &cols,
                        int nrhs, const void *x, int64_t ldx, void *y, int64_t ldy, cdouble alpha,
                        cdouble beta, int maxvals, cudaStream_t st) {
    const bool adj = mode == H2B_ADJOINT;
    if (mode == H2B_FORWARD) {
        if (n.nrow_groups == 0) return cudaSuccess;
        const int bs = block_for(maxvals, 64, 256);
        if (!cplx)
            near_forward_kernel<double><<<n.nrow_groups, bs, 0, st>>>(
                n, rows, cols, nrhs, static_cast<const double *>(x), ldx, static_cast<double *>(y), ldy,
                alpha.x, beta.x, beta.x == 0.0);
        else
            near_forward_kernel<cdouble><<<n.nrow_groups, bs, 0, st>>>(
                n, rows, cols, nrhs, static_cast<const cdouble *>(x), ldx, static_cast<cdouble *>(y), ldy,
                alpha, beta, beta.x == 0.0 && beta.y == 0.0);
        return cudaGetLastError();
    }
    if (n.ncol_groups == 0) return cudaSuccess;
    const int bs = 128;
    cudaError_t err;
    if (!cplx) {
        const size_t sm = (size_t)maxvals * RCH * sizeof(double);
        err = allow_smem(near_transposed_kernel<double>, sm);
        if (err != cudaSuccess) return err;
        near_transposed_kernel<double><<<n.ncol_groups, bs, sm, st>>>(
            n, rows, cols, adj, nrhs, static_cast<const double *>(x), ldx, static_cast<double *>(y), ldy,
            alpha.x, beta.x, beta.x == 0.0);
    } else {
        const size_t sm = (size_t)maxvals * RCH * sizeof(cdouble);
        err = allow_smem(near_transposed_kernel<cdouble>, sm);
        if (err != cudaSuccess) return err;
        near_transposed_kernel<cdouble><<<n.ncol_groups, bs, sm, st>>>(
            n, rows, cols, adj, nrhs, static_cast<const cdouble *>(x), ldx, static_cast<cdouble *>(y), ldy,
            alpha, beta, beta.x == 0.0 && beta.y == 0.0);
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
