/*
 * jci_oracle.c -- CPU restatement of the reference's determinant-CI hot
 * path.  TEST INFRASTRUCTURE ONLY (the checker); the product never links it.
 *
 * Restated from the reference (paths within the reference project):
 *   groups          mpi_source/citruncate.c:121  allocate_eospace_array
 *   string lists    mpi_source/citruncate.c:478  compute_eostrings,
 *                   :3971 generate_string_list   (lexical order per group)
 *   addressing      mpi_source/straddress.c:48   str_adrfind,
 *                   citruncate.c:4093 occstr2address
 *   phases          mpi_source/action_util.c:1462 pindex_single_rep,
 *                   citruncate.c:633 doublerep_cij_yij
 *   validity        citruncate.c:225 check_istring
 *   det order       citruncate.c:414 compute_detnum, pdavidson.c:4757
 *   matrix elems    action_util.c:167 hmatels_0x, :210 hmatels_1x,
 *                   :237 hmatels_2xaa, :250 hmatels_2xab
 *   Davidson        pdavidson.c:39 pdavidson and its helpers (:3773, :3802,
 *                   :4053, :4086, :4821), dsyevr replaced by cyclic Jacobi
 *
 * The excitation enumeration here is generic (every replacement whose
 * result lies in the target group) instead of the reference's 21
 * space-specific generators; the parity tests check that both produce the
 * same set of (index, io, fo, phase) entries.  Sigma is a full-row gather
 * (both triangles), independent of the reference's upper-triangle
 * symmetric accumulation.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "jci_oracle.h"

#define JO_MAXE 20

struct jo_group {
        int docc, actv, virt, nstr, start;
};

struct jo_exc {
        int target;             /* string index */
        int io0, io1, fo0, fo1; /* 1-based orbitals */
        int sign;
};

struct jo_spin {
        int nelec, nstr, ngrp;
        int *istr;                  /* nstr x nelec */
        int *grp;                   /* group of each string */
        struct jo_group *g;
        int *nsing, *ndoub;         /* per-string counts (all groups) */
        long long *osing, *odoub;   /* offsets into lists */
        struct jo_exc *sing, *doub;
};

struct jo_space {
        int norb, ndocc, nactv, xlvl;
        struct jo_spin sp[2];
        int npq;
        int *pq;                    /* npq x 2 */
        int *pairidx;               /* ngrp_a x ngrp_b -> pair or -1 */
        long long *pqoff;           /* det offset of each pair */
        long long ndets;
};

static long long binom(int n, int k)
{
        if (k < 0 || n < 0 || k > n) return 0;
        long long r = 1;
        for (int i = 1; i <= k; i++) r = r * (n - k + i) / i;
        return r;
}

static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }

/* Groups in allocate_eospace_array order (citruncate.c:121-163). */
static int make_groups(int nelec, int norb, int ndocc, int nactv, int xlvl,
                       struct jo_group *g)
{
        int vorbs = norb - ndocc - nactv;
        int mind = ndocc - imin(ndocc, xlvl), maxd = ndocc;
        int mina = (nelec - ndocc) - imin(nelec - ndocc, xlvl);
        int maxa = imin(imin(ndocc, xlvl) + (nelec - ndocc), nactv);
        int n = 0;
        for (int i = maxd; i >= mind; i--)
                for (int j = maxa; j >= mina; j--)
                        for (int k = 0; k <= imin(vorbs, xlvl); k++) {
                                if (i + j + k != nelec) continue;
                                if (g) {
                                        g[n].docc = i;
                                        g[n].actv = j;
                                        g[n].virt = k;
                                }
                                n++;
                        }
        return n;
}

/* Lexical 0-based rank of a sorted relative orbital list r[0..e-1] (values
 * 1..m) among all e-subsets of m orbitals (straddress.c:48-66). */
static long long lex_rank(const int *r, int e, int m)
{
        long long a = 0;
        int prev = 0;
        for (int i = 1; i <= e; i++) {
                for (int j = prev + 1; j <= r[i - 1] - 1; j++)
                        a += binom(m - j, e - i);
                prev = r[i - 1];
        }
        return a;
}

/* Next e-subset of {1..m} in lexical order; returns 0 after the last
 * (straddress.c:106 str_strfind1). */
static int lex_next(int *r, int e, int m)
{
        for (int i = e - 1; i >= 0; i--) {
                if (r[i] < m - (e - 1 - i)) {
                        r[i]++;
                        for (int j = i + 1; j < e; j++) r[j] = r[j - 1] + 1;
                        return 1;
                }
        }
        return 0;
}

static void counts(const struct jo_space *s, const int *o, int ne, int *d,
                   int *a, int *v)
{
        *d = *a = *v = 0;
        for (int i = 0; i < ne; i++) {
                if (o[i] <= s->ndocc) (*d)++;
                else if (o[i] <= s->ndocc + s->nactv) (*a)++;
                else (*v)++;
        }
}

static int find_group(const struct jo_spin *sp, int d, int a, int v)
{
        for (int g = 0; g < sp->ngrp; g++)
                if (sp->g[g].docc == d && sp->g[g].actv == a &&
                    sp->g[g].virt == v)
                        return g;
        return -1;
}

int jo_string_index(const jo_space *s, int spin, const int *o)
{
        const struct jo_spin *sp = &s->sp[spin];
        int ne = sp->nelec, d, a, v;
        for (int i = 1; i < ne; i++)
                if (o[i] <= o[i - 1]) return -1;
        counts(s, o, ne, &d, &a, &v);
        /* check_istring (citruncate.c:225): enough DOCC, few enough VIRT */
        if (d < imax(s->ndocc - s->xlvl, 0) || v > s->xlvl) return -1;
        int g = find_group(sp, d, a, v);
        if (g < 0) return -1;
        int rel[JO_MAXE];
        int vorb = s->norb - s->ndocc - s->nactv;
        for (int i = 0; i < d; i++) rel[i] = o[i];
        long long rd = lex_rank(rel, d, s->ndocc);
        for (int i = 0; i < a; i++) rel[i] = o[d + i] - s->ndocc;
        long long ra = lex_rank(rel, a, s->nactv);
        for (int i = 0; i < v; i++) rel[i] = o[d + a + i] - s->ndocc - s->nactv;
        long long rv = lex_rank(rel, v, vorb);
        long long na = binom(s->nactv, a), nv = binom(vorb, v);
        return (int)(sp->g[g].start + (rd * na + ra) * nv + rv);
}

/* Strings of one group in nested DOCC/ACTV/VIRT lexical order
 * (citruncate.c:478-573), appended at istr[pos*ne]. */
static int emit_group(const struct jo_space *s, int ne, struct jo_group *g,
                      int *istr, int pos)
{
        int vorb = s->norb - s->ndocc - s->nactv;
        int dd[JO_MAXE], aa[JO_MAXE], vv[JO_MAXE];
        int n = 0;
        for (int i = 0; i < g->docc; i++) dd[i] = i + 1;
        do {
                for (int i = 0; i < g->actv; i++) aa[i] = i + 1;
                do {
                        for (int i = 0; i < g->virt; i++) vv[i] = i + 1;
                        do {
                                int *o = istr + (long long)(pos + n) * ne;
                                for (int i = 0; i < g->docc; i++) o[i] = dd[i];
                                for (int i = 0; i < g->actv; i++)
                                        o[g->docc + i] = aa[i] + s->ndocc;
                                for (int i = 0; i < g->virt; i++)
                                        o[g->docc + g->actv + i] =
                                                vv[i] + s->ndocc + s->nactv;
                                n++;
                        } while (g->virt && lex_next(vv, g->virt, vorb));
                } while (g->actv && lex_next(aa, g->actv, s->nactv));
        } while (g->docc && lex_next(dd, g->docc, s->ndocc));
        return n;
}

/* Phase of moving orbital io to fo in the sorted list o (count of occupied
 * orbitals strictly between them; action_util.c:1462). */
static int phase1(const int *o, int ne, int io, int fo)
{
        int lo = io < fo ? io : fo, hi = io < fo ? fo : io, c = 0;
        for (int i = 0; i < ne; i++)
                if (o[i] > lo && o[i] < hi) c++;
        return (c & 1) ? -1 : 1;
}

static void replace_sorted(const int *o, int ne, int io, int fo, int *out)
{
        int n = 0;
        for (int i = 0; i < ne; i++)
                if (o[i] != io) out[n++] = o[i];
        /* insert fo */
        int k = n;
        while (k > 0 && out[k - 1] > fo) {
                out[k] = out[k - 1];
                k--;
        }
        out[k] = fo;
}

static int occupied(const int *o, int ne, int x)
{
        for (int i = 0; i < ne; i++)
                if (o[i] == x) return 1;
        return 0;
}

/* All singles / doubles of string si (any target group). */
static void build_exc(jo_space *s, int spin)
{
        struct jo_spin *sp = &s->sp[spin];
        int ne = sp->nelec, no = s->norb;
        long long cap1 = 0, cap2 = 0;
        sp->nsing = calloc(sp->nstr, sizeof(int));
        sp->ndoub = calloc(sp->nstr, sizeof(int));
        sp->osing = calloc(sp->nstr + 1, sizeof(long long));
        sp->odoub = calloc(sp->nstr + 1, sizeof(long long));
        long long max1 = (long long)ne * (no - ne);
        long long max2 = binom(ne, 2) * binom(no - ne, 2);
        sp->sing = malloc(sizeof(struct jo_exc) * (max1 * sp->nstr + 1));
        sp->doub = malloc(sizeof(struct jo_exc) * (max2 * sp->nstr + 1));
        int t1[JO_MAXE], t2[JO_MAXE];
        for (int si = 0; si < sp->nstr; si++) {
                const int *o = sp->istr + (long long)si * ne;
                sp->osing[si] = cap1;
                sp->odoub[si] = cap2;
                for (int e = 0; e < ne; e++)
                        for (int f = 1; f <= no; f++) {
                                if (occupied(o, ne, f)) continue;
                                replace_sorted(o, ne, o[e], f, t1);
                                int j = jo_string_index(s, spin, t1);
                                if (j < 0) continue;
                                struct jo_exc *x = &sp->sing[cap1++];
                                x->target = j;
                                x->io0 = o[e]; x->io1 = 0;
                                x->fo0 = f; x->fo1 = 0;
                                x->sign = phase1(o, ne, o[e], f);
                        }
                for (int e1 = ne - 1; e1 >= 1; e1--)
                        for (int e2 = e1 - 1; e2 >= 0; e2--)
                                for (int f1 = 1; f1 <= no; f1++) {
                                        if (occupied(o, ne, f1)) continue;
                                        for (int f2 = f1 + 1; f2 <= no; f2++) {
                                                if (occupied(o, ne, f2)) continue;
                                                replace_sorted(o, ne, o[e1], f1, t1);
                                                replace_sorted(t1, ne, o[e2], f2, t2);
                                                int j = jo_string_index(s, spin, t2);
                                                if (j < 0) continue;
                                                struct jo_exc *x = &sp->doub[cap2++];
                                                x->target = j;
                                                x->io0 = o[e1]; x->io1 = o[e2];
                                                x->fo0 = f1; x->fo1 = f2;
                                                x->sign = phase1(o, ne, o[e1], f1) *
                                                          phase1(t1, ne, o[e2], f2);
                                        }
                                }
                sp->nsing[si] = (int)(cap1 - sp->osing[si]);
                sp->ndoub[si] = (int)(cap2 - sp->odoub[si]);
        }
        sp->osing[sp->nstr] = cap1;
        sp->odoub[sp->nstr] = cap2;
}

jo_space *jo_space_build(int ci_aelec, int ci_belec, int ci_orbs, int ndocc,
                         int nactv, int xlvl)
{
        if (ci_aelec > JO_MAXE || ci_belec > JO_MAXE || ci_aelec < 1 ||
            ci_belec < 1 || ndocc + nactv > ci_orbs)
                return NULL;
        jo_space *s = calloc(1, sizeof(*s));
        s->norb = ci_orbs;
        s->ndocc = ndocc;
        s->nactv = nactv;
        s->xlvl = xlvl;
        int ne[2] = {ci_aelec, ci_belec};
        for (int spin = 0; spin < 2; spin++) {
                struct jo_spin *sp = &s->sp[spin];
                sp->nelec = ne[spin];
                sp->ngrp = make_groups(ne[spin], ci_orbs, ndocc, nactv, xlvl,
                                       NULL);
                sp->g = calloc(sp->ngrp + 1, sizeof(struct jo_group));
                make_groups(ne[spin], ci_orbs, ndocc, nactv, xlvl, sp->g);
                int vorb = ci_orbs - ndocc - nactv;
                long long tot = 0;
                for (int g = 0; g < sp->ngrp; g++) {
                        sp->g[g].start = (int)tot;
                        sp->g[g].nstr = (int)(binom(ndocc, sp->g[g].docc) *
                                              binom(nactv, sp->g[g].actv) *
                                              binom(vorb, sp->g[g].virt));
                        tot += sp->g[g].nstr;
                }
                sp->nstr = (int)tot;
                sp->istr = calloc((size_t)tot * ne[spin] + 1, sizeof(int));
                sp->grp = calloc(tot + 1, sizeof(int));
                for (int g = 0; g < sp->ngrp; g++) {
                        emit_group(s, ne[spin], &sp->g[g], sp->istr,
                                   sp->g[g].start);
                        for (int i = 0; i < sp->g[g].nstr; i++)
                                sp->grp[sp->g[g].start + i] = g;
                }
        }
        /* compute_detnum (citruncate.c:414-470) */
        int doccmin = imax(2 * ndocc - xlvl, 0);
        int actvmin = imax((ci_aelec - ndocc) + (ci_belec - ndocc) - xlvl, 0);
        struct jo_spin *P = &s->sp[0], *Q = &s->sp[1];
        s->pq = malloc(sizeof(int) * 2 * (P->ngrp * Q->ngrp + 1));
        s->pairidx = malloc(sizeof(int) * (P->ngrp * Q->ngrp + 1));
        s->pqoff = malloc(sizeof(long long) * (P->ngrp * Q->ngrp + 1));
        s->npq = 0;
        s->ndets = 0;
        for (int i = 0; i < P->ngrp; i++)
                for (int j = 0; j < Q->ngrp; j++) {
                        s->pairidx[i * Q->ngrp + j] = -1;
                        if (P->g[i].docc + Q->g[j].docc < doccmin) continue;
                        if (P->g[i].actv + Q->g[j].actv < actvmin) continue;
                        if (P->g[i].virt + Q->g[j].virt > xlvl) continue;
                        s->pq[2 * s->npq] = i;
                        s->pq[2 * s->npq + 1] = j;
                        s->pairidx[i * Q->ngrp + j] = s->npq;
                        s->pqoff[s->npq] = s->ndets;
                        s->ndets += (long long)P->g[i].nstr * Q->g[j].nstr;
                        s->npq++;
                }
        build_exc(s, 0);
        build_exc(s, 1);
        return s;
}

void jo_space_free(jo_space *s)
{
        if (!s) return;
        for (int spin = 0; spin < 2; spin++) {
                struct jo_spin *sp = &s->sp[spin];
                free(sp->istr); free(sp->grp); free(sp->g);
                free(sp->nsing); free(sp->ndoub); free(sp->osing);
                free(sp->odoub); free(sp->sing); free(sp->doub);
        }
        free(s->pq); free(s->pairidx); free(s->pqoff);
        free(s);
}

void jo_space_info(const jo_space *s, long long *out)
{
        out[0] = s->sp[0].nstr; out[1] = s->sp[1].nstr;
        out[2] = s->sp[0].ngrp; out[3] = s->sp[1].ngrp;
        out[4] = s->npq; out[5] = s->ndets;
}

void jo_strings(const jo_space *s, int spin, int *istr)
{
        const struct jo_spin *sp = &s->sp[spin];
        memcpy(istr, sp->istr, sizeof(int) * (size_t)sp->nstr * sp->nelec);
}

void jo_eospaces(const jo_space *s, int spin, int *out)
{
        const struct jo_spin *sp = &s->sp[spin];
        for (int g = 0; g < sp->ngrp; g++) {
                out[5 * g] = sp->g[g].docc;
                out[5 * g + 1] = sp->g[g].actv;
                out[5 * g + 2] = sp->g[g].virt;
                out[5 * g + 3] = sp->g[g].nstr;
                out[5 * g + 4] = sp->g[g].start;
        }
}

void jo_pq(const jo_space *s, int *out)
{
        memcpy(out, s->pq, sizeof(int) * 2 * s->npq);
}

int jo_excitations(const jo_space *s, int spin, int nrep, int istr,
                   int teosp, int *out)
{
        const struct jo_spin *sp = &s->sp[spin];
        const struct jo_exc *x = nrep == 1 ? sp->sing + sp->osing[istr]
                                           : sp->doub + sp->odoub[istr];
        int n = nrep == 1 ? sp->nsing[istr] : sp->ndoub[istr], c = 0;
        for (int k = 0; k < n; k++) {
                if (sp->grp[x[k].target] != teosp) continue;
                int *o = out + 6 * c++;
                o[0] = x[k].target; o[1] = x[k].io0; o[2] = x[k].io1;
                o[3] = x[k].fo0; o[4] = x[k].fo1; o[5] = x[k].sign;
        }
        return c;
}

/* ---- integrals (moindex.c:14-41) ---------------------------------- */

static long long ix1(int i, int j)
{
        return i > j ? (long long)(i - 1) * i / 2 + j
                     : (long long)(j - 1) * j / 2 + i;
}

static double I1(const double *m1, int i, int j) { return m1[ix1(i, j) - 1]; }

static double I2(const double *m2, int i, int j, int k, int l)
{
        return m2[ix1((int)ix1(i, j), (int)ix1(k, l)) - 1];
}

/* hmatels_0x (action_util.c:167-201) */
static double h0x(const int *a, int na, const int *b, int nb,
                  const double *m1, const double *m2)
{
        double val = 0.0;
        for (int i = 0; i < na; i++) {
                val += I1(m1, a[i], a[i]);
                for (int j = 0; j < i; j++)
                        val += I2(m2, a[i], a[i], a[j], a[j]) -
                               I2(m2, a[i], a[j], a[i], a[j]);
        }
        for (int i = 0; i < nb; i++) {
                val += I1(m1, b[i], b[i]);
                for (int j = 0; j < i; j++)
                        val += I2(m2, b[i], b[i], b[j], b[j]) -
                               I2(m2, b[i], b[j], b[i], b[j]);
        }
        for (int i = 0; i < na; i++)
                for (int j = 0; j < nb; j++)
                        val += I2(m2, a[i], a[i], b[j], b[j]);
        return val;
}

/* hmatels_1x (action_util.c:210-230): s1 is the string being excited. */
static double h1x(const int *s1, int n1, int io, int fo, int pi,
                  const int *s2, int n2, const double *m1, const double *m2)
{
        double val = pi * I1(m1, io, fo);
        for (int i = 0; i < n1; i++)
                if (s1[i] != io)
                        val += pi * (I2(m2, s1[i], s1[i], io, fo) -
                                     I2(m2, s1[i], io, s1[i], fo));
        for (int i = 0; i < n2; i++) val += pi * I2(m2, s2[i], s2[i], io, fo);
        return val;
}

/* hmatels_2xaa (action_util.c:237-245) */
static double h2aa(int i0, int i1, int f0, int f1, int p, const double *m2)
{
        return p * (I2(m2, i0, f0, i1, f1) - I2(m2, i0, f1, i1, f0));
}

/* hmatels_2xab (action_util.c:250-258) */
static double h2ab(int ia, int fa, int pa, int ib, int fb, int pb,
                   const double *m2)
{
        return pa * pb * I2(m2, ia, fa, ib, fb);
}

static void det_strings(const jo_space *s, long long d, int *pp, int *p,
                        int *q)
{
        int k = 0;
        while (k + 1 < s->npq && s->pqoff[k + 1] <= d) k++;
        const struct jo_group *gp = &s->sp[0].g[s->pq[2 * k]];
        const struct jo_group *gq = &s->sp[1].g[s->pq[2 * k + 1]];
        long long r = d - s->pqoff[k];
        *pp = k;
        *p = gp->start + (int)(r / gq->nstr);
        *q = gq->start + (int)(r % gq->nstr);
}

static long long det_index(const jo_space *s, int p, int q)
{
        int gp = s->sp[0].grp[p], gq = s->sp[1].grp[q];
        int k = s->pairidx[gp * s->sp[1].ngrp + gq];
        if (k < 0) return -1;
        return s->pqoff[k] +
               (long long)(p - s->sp[0].g[gp].start) * s->sp[1].g[gq].nstr +
               (q - s->sp[1].g[gq].start);
}

void jo_dyson(const jo_space *s0, const jo_space *s1, int nelec0, int norbs0,
              const double *v0, const double *v1, int nst0, const int *states0,
              int nst1, const int *states1, double *dyorb)
{
        const int sp = nelec0 % 2 == 0 ? 1 : 0;  /* spin that loses the electron */
        const int ne0 = s0->sp[sp].nelec;
        int o[JO_MAXE], r[JO_MAXE];
        memset(dyorb, 0, sizeof(double) * nst0 * nst1 * norbs0);
        for (long long i = 0; i < s0->ndets; i++) {
                int pp, p, q;
                det_strings(s0, i, &pp, &p, &q);
                int x = sp ? q : p;
                memcpy(o, s0->sp[sp].istr + (long long)x * ne0, sizeof(int) * ne0);
                for (int e = 0; e < ne0; e++) {
                        int n = 0;
                        for (int f = 0; f < ne0; f++)
                                if (f != e) r[n++] = o[f];
                        int y = jo_string_index(s1, sp, r);
                        if (y < 0) continue;
                        long long J = sp ? det_index(s1, p, y) : det_index(s1, y, q);
                        if (J < 0) continue;
                        for (int j = 0; j < nst0; j++)
                                for (int k = 0; k < nst1; k++)
                                        dyorb[(j * nst1 + k) * norbs0 + o[e] - 1] +=
                                            v0[(states0[j] - 1) * s0->ndets + i] *
                                            v1[(states1[k] - 1) * s1->ndets + J];
                }
        }
        double pref = sqrt((double)nelec0);
        for (int i = 0; i < nst0 * nst1 * norbs0; i++) dyorb[i] *= pref;
}

void jo_hdiag(const jo_space *s, const double *m1, const double *m2,
              double *out)
{
        int na = s->sp[0].nelec, nb = s->sp[1].nelec;
        for (long long d = 0; d < s->ndets; d++) {
                int k, p, q;
                det_strings(s, d, &k, &p, &q);
                out[d] = h0x(s->sp[0].istr + (long long)p * na, na,
                             s->sp[1].istr + (long long)q * nb, nb, m1, m2);
        }
}

/* Differences of two sorted lists: orbitals in a not in b (ascending). */
static int diff(const int *a, const int *b, int n, int *out)
{
        int c = 0;
        for (int i = 0; i < n; i++)
                if (!occupied(b, n, a[i])) out[c++] = a[i];
        return c;
}

/* Generic Slater-rule element between determinants i and j
 * (action_util.c:119 hmatels and its evaluators). */
double jo_hmatel(const jo_space *s, const double *m1, const double *m2,
                 long long di, long long dj)
{
        int na = s->sp[0].nelec, nb = s->sp[1].nelec;
        int k, pi, qi, pj, qj;
        det_strings(s, di, &k, &pi, &qi);
        det_strings(s, dj, &k, &pj, &qj);
        const int *ai = s->sp[0].istr + (long long)pi * na;
        const int *aj = s->sp[0].istr + (long long)pj * na;
        const int *bi = s->sp[1].istr + (long long)qi * nb;
        const int *bj = s->sp[1].istr + (long long)qj * nb;
        int ax[JO_MAXE], af[JO_MAXE], bx[JO_MAXE], bf[JO_MAXE];
        int nax = diff(ai, aj, na, ax), naf = diff(aj, ai, na, af);
        int nbx = diff(bi, bj, nb, bx), nbf = diff(bj, bi, nb, bf);
        (void)naf; (void)nbf;
        int t1[JO_MAXE];
        if (nax + nbx > 2) return 0.0;
        if (nax + nbx == 0) return h0x(ai, na, bi, nb, m1, m2);
        if (nax == 1 && nbx == 0)
                return h1x(ai, na, ax[0], af[0], phase1(ai, na, ax[0], af[0]),
                           bi, nb, m1, m2);
        if (nax == 0 && nbx == 1)
                return h1x(bi, nb, bx[0], bf[0], phase1(bi, nb, bx[0], bf[0]),
                           ai, na, m1, m2);
        if (nax == 1 && nbx == 1)
                return h2ab(ax[0], af[0], phase1(ai, na, ax[0], af[0]), bx[0],
                            bf[0], phase1(bi, nb, bx[0], bf[0]), m2);
        const int *o = nax == 2 ? ai : bi;
        int n = nax == 2 ? na : nb;
        int *x = nax == 2 ? ax : bx, *f = nax == 2 ? af : bf;
        /* io = (higher, lower), fo ascending, as generate_actvx pairs them */
        replace_sorted(o, n, x[1], f[0], t1);
        int p = phase1(o, n, x[1], f[0]) * phase1(t1, n, x[0], f[1]);
        return h2aa(x[1], x[0], f[0], f[1], p, m2);
}

void jo_sigma(const jo_space *s, const double *m1, const double *m2,
              int nvec, const double *V, double *S)
{
        jo_sigma_range(s, m1, m2, nvec, V, S, 0, s->ndets);
}

/* One sigma row d of nvec vectors into acc[nvec]: the full-row gather of
 * <d|H|j> v_j over every determinant j that differs from d by a single or
 * double replacement (pdavidson.c:1867 compute_hij_eosp and its evaluators
 * :2892-3655, written as a gather instead of the reference's upper-triangle
 * scatter). */
static void sigma_row(const jo_space *s, const double *m1, const double *m2,
                      int nvec, const double *V, long long d, double *acc);

void jo_sigma_range(const jo_space *s, const double *m1, const double *m2,
                    int nvec, const double *V, double *S, long long d0,
                    long long d1)
{
        long long N = s->ndets;
        double *acc = malloc(sizeof(double) * nvec);
        for (long long d = d0; d < d1 && d < N; d++) {
                sigma_row(s, m1, m2, nvec, V, d, acc);
                for (int v = 0; v < nvec; v++) S[v * N + d] = acc[v];
        }
        free(acc);
}

void jo_sigma_rows(const jo_space *s, const double *m1, const double *m2,
                   const double *V, const long long *rows, long long nrows,
                   double *out)
{
        for (long long r = 0; r < nrows; r++) {
                if (rows[r] < 0 || rows[r] >= s->ndets) {
                        out[r] = 0.0;
                        continue;
                }
                sigma_row(s, m1, m2, 1, V, rows[r], &out[r]);
        }
}

static void sigma_row(const jo_space *s, const double *m1, const double *m2,
                      int nvec, const double *V, long long d, double *acc)
{
        const struct jo_spin *A = &s->sp[0], *B = &s->sp[1];
        int na = A->nelec, nb = B->nelec;
        long long N = s->ndets;
        {
                int k, p, q;
                det_strings(s, d, &k, &p, &q);
                const int *sa = A->istr + (long long)p * na;
                const int *sb = B->istr + (long long)q * nb;
                double hd = h0x(sa, na, sb, nb, m1, m2);
                for (int v = 0; v < nvec; v++) acc[v] = hd * V[v * N + d];
                /* alpha singles (same beta) and alpha-beta doubles */
                for (long long x = A->osing[p]; x < A->osing[p + 1]; x++) {
                        const struct jo_exc *e = &A->sing[x];
                        long long j = det_index(s, e->target, q);
                        if (j >= 0) {
                                double h = h1x(sa, na, e->io0, e->fo0, e->sign,
                                               sb, nb, m1, m2);
                                for (int v = 0; v < nvec; v++)
                                        acc[v] += h * V[v * N + j];
                        }
                        for (long long y = B->osing[q]; y < B->osing[q + 1]; y++) {
                                const struct jo_exc *g = &B->sing[y];
                                long long jj = det_index(s, e->target, g->target);
                                if (jj < 0) continue;
                                double h = h2ab(e->io0, e->fo0, e->sign, g->io0,
                                                g->fo0, g->sign, m2);
                                for (int v = 0; v < nvec; v++)
                                        acc[v] += h * V[v * N + jj];
                        }
                }
                for (long long x = A->odoub[p]; x < A->odoub[p + 1]; x++) {
                        const struct jo_exc *e = &A->doub[x];
                        long long j = det_index(s, e->target, q);
                        if (j < 0) continue;
                        double h = h2aa(e->io0, e->io1, e->fo0, e->fo1, e->sign, m2);
                        for (int v = 0; v < nvec; v++) acc[v] += h * V[v * N + j];
                }
                for (long long y = B->osing[q]; y < B->osing[q + 1]; y++) {
                        const struct jo_exc *g = &B->sing[y];
                        long long j = det_index(s, p, g->target);
                        if (j < 0) continue;
                        double h = h1x(sb, nb, g->io0, g->fo0, g->sign, sa, na,
                                       m1, m2);
                        for (int v = 0; v < nvec; v++) acc[v] += h * V[v * N + j];
                }
                for (long long y = B->odoub[q]; y < B->odoub[q + 1]; y++) {
                        const struct jo_exc *g = &B->doub[y];
                        long long j = det_index(s, p, g->target);
                        if (j < 0) continue;
                        double h = h2aa(g->io0, g->io1, g->fo0, g->fo1, g->sign, m2);
                        for (int v = 0; v < nvec; v++) acc[v] += h * V[v * N + j];
                }
        }
}

/* ---- dense eigensolver ------------------------------------------- */

void jo_symeig(int n, double *a, double *w, double *z)
{
        double *v = calloc((size_t)n * n, sizeof(double));
        for (int i = 0; i < n; i++) v[i * n + i] = 1.0;
        for (int sweep = 0; sweep < 100; sweep++) {
                double off = 0.0;
                for (int p = 0; p < n; p++)
                        for (int q = p + 1; q < n; q++) off += a[p * n + q] * a[p * n + q];
                if (off < 1e-30) break;
                for (int p = 0; p < n; p++)
                        for (int q = p + 1; q < n; q++) {
                                double apq = a[p * n + q];
                                if (fabs(apq) < 1e-300) continue;
                                double th = (a[q * n + q] - a[p * n + p]) / (2 * apq);
                                double t = (th >= 0 ? 1.0 : -1.0) /
                                           (fabs(th) + sqrt(th * th + 1.0));
                                double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                                for (int k = 0; k < n; k++) {
                                        double akp = a[k * n + p], akq = a[k * n + q];
                                        a[k * n + p] = c * akp - s * akq;
                                        a[k * n + q] = s * akp + c * akq;
                                }
                                for (int k = 0; k < n; k++) {
                                        double apk = a[p * n + k], aqk = a[q * n + k];
                                        a[p * n + k] = c * apk - s * aqk;
                                        a[q * n + k] = s * apk + c * aqk;
                                }
                                for (int k = 0; k < n; k++) {
                                        double vkp = v[k * n + p], vkq = v[k * n + q];
                                        v[k * n + p] = c * vkp - s * vkq;
                                        v[k * n + q] = s * vkp + c * vkq;
                                }
                        }
        }
        int *ord = malloc(sizeof(int) * n);
        for (int i = 0; i < n; i++) ord[i] = i;
        for (int i = 1; i < n; i++) {
                int t = ord[i], j = i;
                while (j > 0 && a[ord[j - 1] * n + ord[j - 1]] > a[t * n + t]) {
                        ord[j] = ord[j - 1];
                        j--;
                }
                ord[j] = t;
        }
        for (int k = 0; k < n; k++) {
                w[k] = a[ord[k] * n + ord[k]];
                for (int i = 0; i < n; i++) z[k * n + i] = v[i * n + ord[k]];
        }
        free(ord);
        free(v);
}

/* ---- Davidson (pdavidson.c:39-360) -------------------------------- */

static double dot(const double *a, const double *b, long long n)
{
        double s = 0.0;
        for (long long i = 0; i < n; i++) s += a[i] * b[i];
        return s;
}

int jo_davidson(const jo_space *s, const double *m1, const double *m2,
                double totcore, int maxiter, int krymin, int krymax,
                int nroots, int prediagr, int refdim, double restol,
                const double *init, double *energies, double *civec)
{
        long long N = s->ndets;
        if (krymin < nroots || krymax < krymin || N < krymax) return -1;
        double *V = calloc((size_t)krymax * N, sizeof(double));
        double *C = calloc((size_t)krymax * N, sizeof(double));
        double *D = malloc(sizeof(double) * N);
        double *r = malloc(sizeof(double) * N);
        double *t = malloc(sizeof(double) * N);
        double *G = malloc(sizeof(double) * krymax * krymax);
        double *ev = calloc((size_t)krymax * krymax, sizeof(double));
        double *ew = calloc(krymax, sizeof(double));
        double *ov = malloc(sizeof(double) * krymax);
        jo_hdiag(s, m1, m2, D);
        /* build_init_guess_vectors (pdavidson.c:385-452) */
        if (prediagr == 1) {
                if (refdim > N) refdim = (int)N;
                double *h = malloc(sizeof(double) * refdim * refdim);
                double *w = malloc(sizeof(double) * refdim);
                double *z = malloc(sizeof(double) * refdim * refdim);
                for (int i = 0; i < refdim; i++)
                        for (int j = 0; j < refdim; j++)
                                h[i * refdim + j] = jo_hmatel(s, m1, m2, i, j);
                jo_symeig(refdim, h, w, z);
                for (int i = 0; i < krymin; i++)
                        for (int j = 0; j < refdim; j++)
                                V[i * N + j] = i < refdim ? z[i * refdim + j] : 0.0;
                free(h); free(w); free(z);
        } else if (prediagr == 2) {
                for (int i = 0; i < krymin; i++) V[i * N + i] = 1.0;
        } else {
                memcpy(V, init, sizeof(double) * krymin * N);
        }
        int citer = 1, croot = 1, ckdim = krymin, cflag = 0;
        while (citer < maxiter && croot <= nroots) {
                jo_sigma(s, m1, m2, ckdim, V, C);
                for (;;) {
                        /* make_subspacehmat_ga + diag (pdavidson.c:4053,2235):
                         * dsyevr reads the triangle G[i][j] = V_i.C_j, i >= j */
                        for (int i = 0; i < ckdim; i++)
                                for (int j = 0; j <= i; j++) {
                                        double g = dot(V + i * N, C + j * N, N);
                                        G[i * ckdim + j] = G[j * ckdim + i] = g;
                                }
                        double *z = malloc(sizeof(double) * ckdim * ckdim);
                        jo_symeig(ckdim, G, ew, z);
                        for (int i = 0; i < ckdim; i++)
                                for (int j = 0; j < ckdim; j++)
                                        ev[i * krymax + j] = z[i * ckdim + j];
                        free(z);
                        if (ckdim >= krymax) break;
                        /* generate_residual (pdavidson.c:3802) */
                        double th = ew[croot - 1];
                        memset(r, 0, sizeof(double) * N);
                        for (int i = 0; i < ckdim; i++) {
                                double y = ev[(croot - 1) * krymax + i];
                                for (long long d = 0; d < N; d++)
                                        r[d] += y * C[i * N + d] - y * th * V[i * N + d];
                        }
                        double rn = sqrt(dot(r, r, N));
                        /* test_convergence (pdavidson.c:4792) */
                        cflag = rn < restol ? (croot < nroots ? 1 : 2) : 0;
                        if (cflag == 2) break;
                        if (cflag == 1) {
                                croot++;
                                break;
                        }
                        /* generate_newvector: t = r / (theta - D) (:3773) */
                        for (long long d = 0; d < N; d++) t[d] = r[d] / (th - D[d]);
                        /* orthonormalize_newvector: one classical GS pass */
                        for (int i = 0; i < ckdim; i++) ov[i] = dot(V + i * N, t, N);
                        for (int i = 0; i < ckdim; i++)
                                for (long long d = 0; d < N; d++)
                                        t[d] -= ov[i] * V[i * N + d];
                        double nn = 1.0 / sqrt(dot(t, t, N));
                        for (long long d = 0; d < N; d++) t[d] *= nn;
                        memcpy(V + ckdim * N, t, sizeof(double) * N);
                        jo_sigma(s, m1, m2, 1, t, C + ckdim * N);
                        ckdim++;
                        citer++;
                }
                /* truncate_krylov_space (pdavidson.c:4821): V <- V Y[:, :krymin] */
                double *X = calloc((size_t)krymin * N, sizeof(double));
                for (int i = 0; i < krymin; i++)
                        for (int j = 0; j < ckdim; j++) {
                                double y = ev[i * krymax + j];
                                for (long long d = 0; d < N; d++)
                                        X[i * N + d] += y * V[j * N + d];
                        }
                memset(V, 0, sizeof(double) * krymax * N);
                memcpy(V, X, sizeof(double) * krymin * N);
                free(X);
                memset(C, 0, sizeof(double) * krymax * N);
                ckdim = krymin;
                if (cflag == 2) break;
        }
        for (int i = 0; i < nroots; i++) energies[i] = ew[i] + totcore;
        if (civec) memcpy(civec, V, sizeof(double) * nroots * N);
        free(V); free(C); free(D); free(r); free(t); free(G);
        free(ev); free(ew); free(ov);
        return citer;
}
