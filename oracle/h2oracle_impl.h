/*
 * Body of the CPU oracle, included once per scalar type by h2oracle.c with
 *   SC       scalar type (double or double _Complex)
 *   CONJ(z)  complex conjugate (identity for real scalars)
 *   SFX(n)   name suffix
 *
 * This is TEST INFRASTRUCTURE: the plain CPU restatement of H2Factory.jl's matvec that the CUDA
 * library is checked against. It is not part of the product path.
 *
 * Every step follows the reference's per-node traversal, including its overwrite/accumulate
 * order, so that the GPU kernels can be compared against the same arithmetic:
 *   aggregatetree!                src/farinteractions/aggregation.jl:58-134, :241-272
 *   disaggregatetranslatetree!    src/farinteractions/disaggregation.jl:106-295
 *   translateintonode!            src/farinteractions/traversalhelpers.jl:167-219
 *   leaf products                 src/moments/create/linkmomenttocollection.jl:56-63, :386-411
 *   adjoint leaf products         src/maps/functors.jl:227-259
 *   level transfers               src/maps/leveltranslator.jl:122-265
 *   dense / diagonal couplings    src/farinteractions/i2otranslations/i2otranslationcollection.jl:367-495
 *   Toeplitz couplings            src/moments/toeplitz/toeplitzmul.jl:95-315,
 *                                 src/farinteractions/i2otranslations/toeplitzi2ocollection.jl:109-272
 *   near product                  src/nearinteractions/nearmul.jl:8-14 (SparseMatrixCSC mul!)
 */

/* Moments of one side, one slot per node: [comp][rhs][coef]. */
typedef struct {
    SC *m;            /* ordinary moments */
    int64_t *off;     /* [nnodes] element offset, -1 if the node has no slot */
    double _Complex *t; /* Toeplitz padded arrays, [comp][rhs][tsize] per node */
    int64_t *toff;
} SFX(momentstore);

static int64_t SFX(ncoef)(const h2b_side_desc *s, int lvl) {
    return (int64_t)s->shape[3 * lvl] * s->shape[3 * lvl + 1] * s->shape[3 * lvl + 2];
}

static int64_t SFX(tsize)(const h2b_side_desc *s, int lvl) {
    int64_t t = 1;
    for (int d = 0; d < 3; ++d) t *= 2 * (int64_t)s->shape[3 * lvl + d] - 1;
    return t;
}

static int SFX(isleaf)(const h2b_side_desc *s, int n) { return s->child_ptr[n + 1] == s->child_ptr[n]; }

static int SFX(alloc_store)(const h2b_map_desc *d, const h2b_side_desc *s, int nrhs, int toeplitz,
                            SFX(momentstore) * st) {
    st->off = (int64_t *)malloc(sizeof(int64_t) * (size_t)s->nnodes);
    st->toff = (int64_t *)malloc(sizeof(int64_t) * (size_t)s->nnodes);
    if (!st->off || !st->toff) return 0;
    int64_t total = 0, ttotal = 0;
    for (int n = 0; n < s->nnodes; ++n) {
        st->off[n] = total;
        st->toff[n] = ttotal;
        total += (int64_t)d->ncomp * nrhs * SFX(ncoef)(s, s->level[n]);
        if (toeplitz) ttotal += (int64_t)d->ncomp * nrhs * SFX(tsize)(s, s->level[n]);
    }
    st->m = (SC *)calloc((size_t)(total > 0 ? total : 1), sizeof(SC));
    st->t = (double _Complex *)calloc((size_t)(ttotal > 0 ? ttotal : 1), sizeof(double _Complex));
    return st->m && st->t;
}

static void SFX(free_store)(SFX(momentstore) * st) {
    free(st->m);
    free(st->off);
    free(st->t);
    free(st->toff);
}

/* ---------------------------------------------------------------------------------------------
 * Leaf products.
 * Aggregation, mul!(moment, coll, x): moment[i] = coll[i] * x  (linkmomenttocollection.jl:56-63);
 * adjoint with ConjugatedCollectionMul: conj(coll[i]) * x       (functors.jl:231-238).
 * ------------------------------------------------------------------------------------------- */
static void SFX(leaf_aggregate)(const h2b_map_desc *d, const h2b_side_desc *s, int node, int conjc,
                                int nrhs, const SC *x, int64_t ldx, SC *mom) {
    const int64_t nc = SFX(ncoef)(s, s->level[node]);
    const int32_t v0 = s->value_ptr[node], nv = s->value_ptr[node + 1] - v0;
    const SC *coll = (const SC *)s->coll + s->coll_offset[node];
    for (int c = 0; c < d->ncomp; ++c) {
        const SC *C = coll + (int64_t)c * nc * nv;
        for (int r = 0; r < nrhs; ++r) {
            SC *m = mom + ((int64_t)c * nrhs + r) * nc;
            for (int64_t a = 0; a < nc; ++a) m[a] = 0;
            for (int j = 0; j < nv; ++j) {
                const SC xj = x[(int64_t)r * ldx + s->value[v0 + j]];
                for (int64_t a = 0; a < nc; ++a) {
                    const SC cij = C[a + (int64_t)j * nc];
                    m[a] += (conjc ? CONJ(cij) : cij) * xj;
                }
            }
        }
    }
}

/* Disaggregation, mul!(y, coll, moment, α, β): y = α Σ_i transpose(coll[i]) m[i] + β y, with β on
 * the first component only (linkmomenttocollection.jl:386-411); adjoint collections use
 * adjoint(coll[i]) (functors.jl:240-259). β == 0 overwrites, as LinearAlgebra.mul! does. */
static void SFX(leaf_disaggregate)(const h2b_map_desc *d, const h2b_side_desc *s, int node,
                                   int conjc, int nrhs, const SC *mom, SC alpha, SC beta,
                                   SC *y, int64_t ldy) {
    const int64_t nc = SFX(ncoef)(s, s->level[node]);
    const int32_t v0 = s->value_ptr[node], nv = s->value_ptr[node + 1] - v0;
    const SC *coll = (const SC *)s->coll + s->coll_offset[node];
    for (int r = 0; r < nrhs; ++r) {
        for (int j = 0; j < nv; ++j) {
            SC acc = 0;
            for (int c = 0; c < d->ncomp; ++c) {
                const SC *C = coll + (int64_t)c * nc * nv + (int64_t)j * nc;
                const SC *m = mom + ((int64_t)c * nrhs + r) * nc;
                SC part = 0;
                for (int64_t a = 0; a < nc; ++a) part += (conjc ? CONJ(C[a]) : C[a]) * m[a];
                acc += alpha * part;
            }
            SC *yj = &y[(int64_t)r * ldy + s->value[v0 + j]];
            *yj = (beta == 0) ? acc : acc + beta * *yj;
        }
    }
}

/* ---------------------------------------------------------------------------------------------
 * Level transfers: out (+)= op(T) in, op per applytransfer! direction
 * (leveltranslator.jl:122-158): 0 forward, 1 transpose, 2 adjoint, 3 conjugate.
 * ------------------------------------------------------------------------------------------- */
static SC SFX(opentry)(const SC *T, int64_t ldt, int64_t i, int64_t j, int op) {
    /* entry (i, j) of op(T), T column-major with leading dimension ldt */
    switch (op) {
    case 0: return T[i + j * ldt];
    case 3: return CONJ(T[i + j * ldt]);
    case 1: return T[j + i * ldt];
    default: return CONJ(T[j + i * ldt]);
    }
}

static void SFX(dense_apply)(const SC *T, int64_t ldt, int64_t nout, int64_t nin, int op,
                             const SC *in, SC *out, int accumulate) {
    for (int64_t i = 0; i < nout; ++i) {
        SC acc = 0;
        for (int64_t j = 0; j < nin; ++j) acc += SFX(opentry)(T, ldt, i, j, op) * in[j];
        out[i] = accumulate ? out[i] + acc : acc;
    }
}

/* Separable contraction, axes from `dim` down to 1 (_applyonedimseparable!,
 * leveltranslator.jl:200-265). `fin`/`fout` are the moment extents on the in/out side. */
static void SFX(separable_apply)(const SC *const *M, const int64_t *ldm, int dim, const int *fin,
                                 const int *fout, int op, const SC *in, SC *out, int accumulate) {
    int cur[3] = {fin[0], fin[1], fin[2]};
    int64_t maxlen = 1;
    for (int dd = 0; dd < 3; ++dd) maxlen *= (fin[dd] > fout[dd] ? fin[dd] : fout[dd]);
    SC *a = (SC *)malloc(sizeof(SC) * (size_t)maxlen);
    SC *b = (SC *)malloc(sizeof(SC) * (size_t)maxlen);
    int64_t len = (int64_t)fin[0] * fin[1] * fin[2];
    for (int64_t k = 0; k < len; ++k) a[k] = in[k];
    for (int ax = dim - 1; ax >= 0; --ax) {
        int nxt[3] = {cur[0], cur[1], cur[2]};
        nxt[ax] = fout[ax];
        /* op(M_ax) is fout[ax] x fin[ax] */
        for (int i3 = 0; i3 < nxt[2]; ++i3)
            for (int i2 = 0; i2 < nxt[1]; ++i2)
                for (int i1 = 0; i1 < nxt[0]; ++i1) {
                    int idx[3] = {i1, i2, i3};
                    int row = idx[ax];
                    SC acc = 0;
                    for (int k = 0; k < cur[ax]; ++k) {
                        int src[3] = {i1, i2, i3};
                        src[ax] = k;
                        acc += SFX(opentry)(M[ax], ldm[ax], row, k, op) *
                               a[src[0] + (int64_t)cur[0] * (src[1] + (int64_t)cur[1] * src[2])];
                    }
                    b[i1 + (int64_t)nxt[0] * (i2 + (int64_t)nxt[1] * i3)] = acc;
                }
        cur[0] = nxt[0]; cur[1] = nxt[1]; cur[2] = nxt[2];
        SC *tmp = a; a = b; b = tmp;
    }
    len = (int64_t)fout[0] * fout[1] * fout[2];
    for (int64_t k = 0; k < len; ++k) out[k] = accumulate ? out[k] + a[k] : a[k];
    free(a);
    free(b);
}

/* Apply the (level(child), sector(child)) transfer of side `s` between parent and child slots. */
static void SFX(transfer)(const h2b_map_desc *d, const h2b_side_desc *s, int child, int op,
                          int nrhs, const SC *in, SC *out, int accumulate) {
    const int lc = s->level[child], lp = lc - 1;
    const int64_t toff = s->transfer_offset[(int64_t)lc * d->nsectors + s->sector[child]];
    const SC *T = (const SC *)s->transfer + toff;
    const int upward = (op == 0 || op == 3);
    const int *sin_ = upward ? &s->shape[3 * lc] : &s->shape[3 * lp];
    const int *sout = upward ? &s->shape[3 * lp] : &s->shape[3 * lc];
    const int64_t nin = (int64_t)sin_[0] * sin_[1] * sin_[2];
    const int64_t nout = (int64_t)sout[0] * sout[1] * sout[2];
    for (int c = 0; c < d->ncomp; ++c)
        for (int r = 0; r < nrhs; ++r) {
            const SC *vi = in + ((int64_t)c * nrhs + r) * nin;
            SC *vo = out + ((int64_t)c * nrhs + r) * nout;
            if (d->transfer_kind == H2B_TRANSFER_DENSE) {
                /* stored T is ncoef(parent) x ncoef(child) */
                const int64_t ldt = SFX(ncoef)(s, lp);
                SFX(dense_apply)(T, ldt, nout, nin, op, vi, vo, accumulate);
            } else {
                const SC *M[3];
                int64_t ldm[3];
                int64_t o = 0;
                for (int ax = 0; ax < d->dim; ++ax) {
                    M[ax] = T + o;
                    ldm[ax] = s->shape[3 * lp + ax];
                    o += (int64_t)s->shape[3 * lp + ax] * s->shape[3 * lc + ax];
                }
                SFX(separable_apply)(M, ldm, d->dim, sin_, sout, op, vi, vo, accumulate);
            }
        }
}

/* ---------------------------------------------------------------------------------------------
 * FFT of the padded Toeplitz arrays. AbstractFFTs conventions: fft unnormalised with e^{-2πi jk/n},
 * ifft with e^{+2πi jk/n} and 1/n per axis (toeplitzmul.jl:290-315). Plain DFT per axis.
 * ------------------------------------------------------------------------------------------- */
static void SFX(dft_axes)(double _Complex *a, const int *ts, int inverse) {
    double _Complex line[64], outl[64], tw[64];
    for (int ax = 0; ax < 3; ++ax) {
        const int n = ts[ax];
        if (n == 1) continue;
        /* the twiddle of (j, k) depends on j k mod n only: one table per axis (an FFTW plan's role,
           ext/H2Toeplitz/toeplitzi2ocollection.jl:34-58), the same values the direct sum used */
        for (int m = 0; m < n; ++m) {
            const double ang = (inverse ? 2.0 : -2.0) * M_PI * (double)m / n;
            tw[m] = cos(ang) + I * sin(ang);
        }
        const int64_t stride = ax == 0 ? 1 : (ax == 1 ? ts[0] : (int64_t)ts[0] * ts[1]);
        const int64_t total = (int64_t)ts[0] * ts[1] * ts[2];
        for (int64_t base = 0; base < total; ++base) {
            /* visit each line once: base must have coordinate 0 along ax */
            if ((base / stride) % n != 0) continue;
            for (int k = 0; k < n; ++k) line[k] = a[base + k * stride];
            for (int k = 0; k < n; ++k) {
                double _Complex acc = 0;
                for (int j = 0; j < n; ++j) acc += line[j] * tw[(int64_t)j * k % n];
                outl[k] = inverse ? acc / n : acc;
            }
            for (int k = 0; k < n; ++k) a[base + k * stride] = outl[k];
        }
    }
}

/* modulate_in!: zero the padded array, copy the moment into its leading corner, transform. */
static void SFX(modulate_in)(const h2b_map_desc *d, const h2b_side_desc *s, int node, int inverse,
                             int nrhs, const SC *mom, double _Complex *spec) {
    const int lvl = s->level[node];
    const int *sh = &s->shape[3 * lvl];
    int ts[3] = {2 * sh[0] - 1, 2 * sh[1] - 1, 2 * sh[2] - 1};
    const int64_t nt = (int64_t)ts[0] * ts[1] * ts[2], nc = (int64_t)sh[0] * sh[1] * sh[2];
    for (int q = 0; q < d->ncomp * nrhs; ++q) {
        double _Complex *t = spec + q * nt;
        const SC *m = mom + q * nc;
        for (int64_t k = 0; k < nt; ++k) t[k] = 0;
        for (int i3 = 0; i3 < sh[2]; ++i3)
            for (int i2 = 0; i2 < sh[1]; ++i2)
                for (int i1 = 0; i1 < sh[0]; ++i1)
                    t[i1 + ts[0] * ((int64_t)i2 + ts[1] * i3)] = m[i1 + sh[0] * ((int64_t)i2 + sh[1] * i3)];
        SFX(dft_axes)(t, ts, inverse);
    }
}

/* modulate_out!: transform back and copy the leading corner into the moment (overwrite). */
static void SFX(modulate_out)(const h2b_map_desc *d, const h2b_side_desc *s, int node, int inverse,
                              int nrhs, double _Complex *spec, SC *mom) {
    const int lvl = s->level[node];
    const int *sh = &s->shape[3 * lvl];
    int ts[3] = {2 * sh[0] - 1, 2 * sh[1] - 1, 2 * sh[2] - 1};
    const int64_t nt = (int64_t)ts[0] * ts[1] * ts[2], nc = (int64_t)sh[0] * sh[1] * sh[2];
    for (int q = 0; q < d->ncomp * nrhs; ++q) {
        double _Complex *t = spec + q * nt;
        SC *m = mom + q * nc;
        SFX(dft_axes)(t, ts, inverse);
        for (int i3 = 0; i3 < sh[2]; ++i3)
            for (int i2 = 0; i2 < sh[1]; ++i2)
                for (int i1 = 0; i1 < sh[0]; ++i1)
                    m[i1 + sh[0] * ((int64_t)i2 + sh[1] * i3)] =
                        TAKEREAL(t[i1 + ts[0] * ((int64_t)i2 + ts[1] * i3)]);
    }
}

/* ---------------------------------------------------------------------------------------------
 * The far product (farmul!, src/farinteractions/farmul.jl:47-70).
 * ------------------------------------------------------------------------------------------- */
static int SFX(farmul)(const h2b_map_desc *d, int mode, int nrhs, const SC *x, int64_t ldx, SC *y,
                       int64_t ldy, const double *alpha, const double *beta) {
    const h2b_side_desc *as = (mode == H2B_FORWARD) ? &d->trial : &d->test;
    const h2b_side_desc *ds = (mode == H2B_FORWARD) ? &d->test : &d->trial;
    const int toeplitz = d->coupling_kind == H2B_COUPLING_TOEPLITZ;
    /* aggregationdirection / disaggregationdirection / translationdirection
       (translationcontext.jl:57-59, accessors.jl:409-416, :370-381) */
    const int i2iop = (mode == H2B_ADJOINT) ? 3 : 0;
    const int o2oop = (mode == H2B_ADJOINT) ? 2 : 1;
    const int i2oop = mode; /* 0 forward, 1 transpose, 2 adjoint */
    const int conjc = (mode == H2B_ADJOINT) && d->conj_leaf_adjoint;
    /* Toeplitz plan order: transpose swaps fft and ifft (toeplitzi2ocollection.jl:248-272) */
    const int in_inverse = (mode == H2B_TRANSPOSE), out_inverse = (mode != H2B_TRANSPOSE);
    SC alphaA = (SC)d->alpha[mode][0] MKIMAG(d->alpha[mode][1]);

    SFX(momentstore) am, dm;
    if (!SFX(alloc_store)(d, as, nrhs, toeplitz, &am) || !SFX(alloc_store)(d, ds, nrhs, toeplitz, &dm)) {
        oracle_set_error("out of host memory");
        return H2B_ERR_NOMEM;
    }

    /* ---- aggregate! (aggregation.jl:58-134, :241-272) ---- */
    for (int st = 0; st < as->agg_nstages; ++st) {
        const int lo = as->agg_ptr[st], hi = as->agg_ptr[st + 1];
#pragma omp parallel for schedule(dynamic, 8)
        for (int k = lo; k < hi; ++k) {
            const int node = as->agg_node[k];
            if (SFX(isleaf)(as, node))
                SFX(leaf_aggregate)(d, as, node, conjc, nrhs, x, ldx, am.m + am.off[node]);
        }
#pragma omp parallel for schedule(dynamic, 8)
        for (int k = lo; k < hi; ++k) {
            const int node = as->agg_node[k];
            if (!SFX(isleaf)(as, node)) {
                /* i2ipass!: first child overwrites, the rest accumulate (traversalhelpers.jl:49-75) */
                for (int q = as->child_ptr[node]; q < as->child_ptr[node + 1]; ++q) {
                    const int ch = as->child[q];
                    SFX(transfer)(d, as, ch, i2iop, nrhs, am.m + am.off[ch], am.m + am.off[node],
                                  q != as->child_ptr[node]);
                }
            }
            if (toeplitz && as->agg_store[node])
                SFX(modulate_in)(d, as, node, in_inverse, nrhs, am.m + am.off[node], am.t + am.toff[node]);
        }
    }

    /* ---- disaggregate! (disaggregation.jl:106-295) ---- */
    SC salpha = (SC)alpha[0] MKIMAG(alpha[1]);
    SC sbeta = (SC)beta[0] MKIMAG(beta[1]);
    for (int st = 0; st < ds->dis_nstages; ++st) {
        const int lo = ds->dis_ptr[st], hi = ds->dis_ptr[st + 1];
#pragma omp parallel for schedule(dynamic, 8)
        for (int k = lo; k < hi; ++k) {
            const int node = ds->dis_node[k];
            const int lvl = ds->level[node];
            const int64_t nc = SFX(ncoef)(ds, lvl);
            SC *out = dm.m + dm.off[node];
            int initialized = 0;
            /* translateintonode! (traversalhelpers.jl:167-219) */
            for (int p = ds->i2o_ptr[node]; p < ds->i2o_ptr[node + 1]; ++p) {
                const int src = ds->i2o_src[p];
                const int slvl = as->level[src];
                const int64_t snc = SFX(ncoef)(as, slvl);
                const int64_t key = ds->i2o_coupling[p];
                const int64_t coff = d->coupling_offset[key];
                /* symmetry-reduced couplings: canonical data read through permutations */
                const int32_t *rp = (d->coupling_rowperm && d->coupling_rowperm[key] >= 0)
                                        ? d->coupling_perm + d->coupling_rowperm[key] : NULL;
                const int32_t *cp = (d->coupling_colperm && d->coupling_colperm[key] >= 0)
                                        ? d->coupling_perm + d->coupling_colperm[key] : NULL;
                if (d->coupling_kind == H2B_COUPLING_DENSE) {
                    /* mul!(out, op(block), in[, true, true]), i2otranslationcollection.jl:367-409.
                       The stored block of the resolved key is ncoef(key recv) x ncoef(key transl). */
                    const SC *B = (const SC *)(d->coupling + coff);
                    const int64_t ldb = (i2oop == 0) ? nc : snc;
                    for (int q = 0; q < d->ncomp * nrhs; ++q) {
                        const SC *in = am.m + am.off[src] + q * snc;
                        SC *o = out + q * nc;
                        if (!rp && !cp) {
                            SFX(dense_apply)(B, ldb, nc, snc, i2oop, in, o, initialized);
                            continue;
                        }
                        /* PermutedDenseTranslation: gather the input, multiply by the canonical
                           block, scatter the output; transposed maps gather with the row and
                           scatter with the column permutation (symmetryreduceddense.jl:84-95) */
                        const int32_t *gp = (i2oop == 0) ? cp : rp, *sp = (i2oop == 0) ? rp : cp;
                        SC *w = (SC *)malloc(sizeof(SC) * (size_t)(snc + nc));
                        SC *yv = w + snc;
                        for (int64_t j = 0; j < snc; ++j) w[j] = in[gp ? gp[j] : j];
                        SFX(dense_apply)(B, ldb, nc, snc, i2oop, w, yv, 0);
                        for (int64_t i = 0; i < nc; ++i) {
                            const int64_t k = sp ? sp[i] : i;
                            o[k] = initialized ? o[k] + yv[i] : yv[i];
                        }
                        free(w);
                    }
                } else if (d->coupling_kind == H2B_COUPLING_DIAGONAL) {
                    /* elementwisemul!, adjoint conjugates (i2otranslationcollection.jl:415-495) */
                    const SC *D = (const SC *)(d->coupling + coff);
                    for (int q = 0; q < d->ncomp * nrhs; ++q)
                        for (int64_t a = 0; a < nc; ++a) {
                            const SC v = (i2oop == 2 ? CONJ(D[a]) : D[a]) * am.m[am.off[src] + q * snc + a];
                            out[q * nc + a] = initialized ? out[q * nc + a] + v : v;
                        }
                } else {
                    /* toeplitzmul! / adjointtoeplitzmul! (toeplitzmul.jl:95-100, :265-288) */
                    const double _Complex *K = (const double _Complex *)(d->coupling + coff);
                    const int64_t nt = SFX(tsize)(ds, lvl);
                    double _Complex *tout = dm.t + dm.toff[node];
                    const double _Complex *tin = am.t + am.toff[src];
                    for (int q = 0; q < d->ncomp * nrhs; ++q)
                        for (int64_t e = 0; e < nt; ++e) {
                            /* PermutedTranslation: t[e] = canonical[perm[e]] */
                            const double _Complex ke = K[rp ? rp[e] : e];
                            const double _Complex kv = (i2oop == 2) ? conj(ke) : ke;
                            const double _Complex v = kv * tin[q * nt + e];
                            tout[q * nt + e] = initialized ? tout[q * nt + e] + v : v;
                        }
                }
                initialized = 1;
            }
            if (initialized && toeplitz)
                SFX(modulate_out)(d, ds, node, out_inverse, nrhs, dm.t + dm.toff[node], out);
            /* O2O from the parent (disaggregation.jl:244-271) */
            if (node != ds->root) {
                const int parent = ds->parent[node];
                if (ds->dis_isnode[parent]) {
                    SFX(transfer)(d, ds, node, o2oop, nrhs, dm.m + dm.off[parent], out, initialized);
                    initialized = 1;
                }
            }
        }
        /* leaf scatter after the stage (disaggregateleafchunk!, traversalhelpers.jl:140-158),
           for leaves with hasinitializedmoment (traversalhelpers.jl:103-112) */
#pragma omp parallel for schedule(dynamic, 8)
        for (int k = lo; k < hi; ++k) {
            const int node = ds->dis_node[k];
            if (!SFX(isleaf)(ds, node)) continue;
            int init = ds->i2o_ptr[node + 1] > ds->i2o_ptr[node];
            if (node != ds->root && ds->dis_isnode[ds->parent[node]]) init = 1;
            if (!init) continue;
            SFX(leaf_disaggregate)(d, ds, node, conjc, nrhs, dm.m + dm.off[node], alphaA * salpha,
                                   sbeta, y, ldy);
        }
    }
    SFX(free_store)(&am);
    SFX(free_store)(&dm);
    return H2B_OK;
}

/* ---------------------------------------------------------------------------------------------
 * Near product: y = α op(N) x + β y with the SparseMatrixCSC rule: β scales (or, when zero,
 * clears) all of y first, then α N x is added (nearmul.jl:8-14, accessors.jl:149-159).
 * Blocks are grouped by the leaf that owns their output rows, so output leaves run in parallel.
 * ------------------------------------------------------------------------------------------- */
static int SFX(nearmul)(const h2b_map_desc *d, int mode, int nrhs, const SC *x, int64_t ldx, SC *y,
                        int64_t ldy, SC alpha, SC beta) {
    const h2b_side_desc *rs = &d->test, *cs = &d->trial;
    const h2b_side_desc *os = (mode == H2B_FORWARD) ? rs : cs;
    const int64_t ny = os->ndofs;
    for (int r = 0; r < nrhs; ++r)
        for (int64_t i = 0; i < ny; ++i) {
            SC *v = &y[(int64_t)r * ldy + i];
            *v = (beta == 0) ? 0 : beta * *v;
        }
    const int nb = d->near_nrows > 0 ? d->near_ptr[d->near_nrows] : 0;
    int *brow = (int *)malloc(sizeof(int) * (size_t)(nb + 1));
    int *ptr = (int *)calloc((size_t)os->nnodes + 1, sizeof(int));
    int *order = (int *)malloc(sizeof(int) * (size_t)(nb + 1));
    if (!brow || !ptr || !order) { free(brow); free(ptr); free(order); oracle_set_error("out of host memory"); return H2B_ERR_NOMEM; }
    for (int g = 0; g < d->near_nrows; ++g)
        for (int b = d->near_ptr[g]; b < d->near_ptr[g + 1]; ++b) brow[b] = d->near_row[g];
    for (int b = 0; b < nb; ++b) ptr[(mode == H2B_FORWARD ? brow[b] : d->near_col[b]) + 1]++;
    for (int n = 0; n < os->nnodes; ++n) ptr[n + 1] += ptr[n];
    {
        int *fill = (int *)malloc(sizeof(int) * (size_t)(os->nnodes + 1));
        memcpy(fill, ptr, sizeof(int) * (size_t)(os->nnodes + 1));
        for (int b = 0; b < nb; ++b) order[fill[mode == H2B_FORWARD ? brow[b] : d->near_col[b]]++] = b;
        free(fill);
    }
    const SC *N = (const SC *)d->near;
#pragma omp parallel for schedule(dynamic, 4)
    for (int leaf = 0; leaf < os->nnodes; ++leaf) {
        for (int k = ptr[leaf]; k < ptr[leaf + 1]; ++k) {
            const int b = order[k];
            const int row = brow[b], col = d->near_col[b];
            const int r0 = rs->value_ptr[row], nr = rs->value_ptr[row + 1] - r0;
            const int c0 = cs->value_ptr[col], nc = cs->value_ptr[col + 1] - c0;
            const SC *B = N + d->near_offset[b];
            for (int q = 0; q < nrhs; ++q) {
                const SC *xq = x + (int64_t)q * ldx;
                SC *yq = y + (int64_t)q * ldy;
                if (mode == H2B_FORWARD) {
                    for (int j = 0; j < nc; ++j) {
                        const SC ax = alpha * xq[cs->value[c0 + j]];
                        for (int i = 0; i < nr; ++i) yq[rs->value[r0 + i]] += B[i + (int64_t)j * nr] * ax;
                    }
                } else {
                    const int cj = (mode == H2B_ADJOINT);
                    for (int j = 0; j < nc; ++j) {
                        SC acc = 0;
                        for (int i = 0; i < nr; ++i) {
                            const SC bij = B[i + (int64_t)j * nr];
                            acc += (cj ? CONJ(bij) : bij) * xq[rs->value[r0 + i]];
                        }
                        yq[cs->value[c0 + j]] += alpha * acc;
                    }
                }
            }
        }
    }
    free(brow);
    free(ptr);
    free(order);
    return H2B_OK;
}
