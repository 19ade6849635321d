/*
 * forest.c - adaptive quadtree / octree meshes on the host: the role the
 * p4est forest (DMP4EST / DMP8EST, "brick" topology) plays for the reference
 * (created in src/cipher.c:1149-1159, adapted in src/cipher.c:1365-1586 and
 * 1607-1829), linearised to leaf arrays.
 *
 * A forest covers nb[0] x nb[1] (x nb[2]) blocks; a leaf of level l is a
 * square / cube of 2^(lmax-l) finest cells, so the finest grid has
 * res[d] = nb[d] * 2^lmax cells.  Leaves are kept in brick order: blocks x
 * fastest, and inside a block the Morton (z-order) order of the leaves'
 * lower corners, which lists the children of a node consecutively.
 *
 * Adaptation follows the reference's use of DMAdaptLabel: a leaf marked
 * refine splits once (up to lmax), a family of 2^dim siblings all marked
 * coarsen merges into its parent (down to lmin), everything else stays;
 * then 2:1 balance across faces refines leaves that are more than one level
 * coarser than a face neighbour, repeatedly.  The finite-volume transfer of
 * a state (DMForestTransferVec) copies a leaf's dofs into its children and
 * averages a coarsened family's dofs into the parent.  A family whose active
 * sets differ is not coarsened (an average of phase ids is no phase id).
 *
 * The mesh of a forest (cipher_forest_mesh) lists the leaves as cells with
 * cellgeom = vol^(1/dim), every interior face once - conforming faces and
 * the hanging faces between a coarse leaf and each of its finer neighbours,
 * which the reference's face loop visits as separate faces
 * (src/cipher.c:1208-1225: support-2 faces without children) - and the
 * boundary faces of non-periodic sides with the reference's labels
 * (src/cipher.c:1212-1220).  Face order: by the lower (L) cell, then the
 * direction, then the neighbour's leaf index.
 */
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "cipher_problem.h"
#include "cipher_b200.h"

typedef struct {
    int32_t level;
    int32_t c[3];       /* lower corner on the finest grid */
} fleaf;

struct cipher_forest {
    int dim, lmin, lmax;
    int32_t nb[3], res[3], periodic[3];
    double size[3];
    int64_t n;
    fleaf *leaf;
    /* transfer plan of the last adaptation: new leaf i takes the mean of old
     * leaves [src0[i], src0[i] + nsrc[i]) (NULL before the first) */
    int64_t n_old;
    int64_t *src0;
    int32_t *nsrc;
};

static int32_t side_of(const cipher_forest *f, int level) { return (int32_t)1 << (f->lmax - level); }

/* brick order key: block index, then the Morton code of the corner inside the block */
static uint64_t leaf_key(const cipher_forest *f, const fleaf *L)
{
    uint64_t blk = 0, mul = 1;
    for (int d = 0; d < f->dim; d++) {
        blk += (uint64_t)(L->c[d] >> f->lmax) * mul;
        mul *= (uint64_t)f->nb[d];
    }
    uint64_t m = 0;
    const int32_t mask = ((int32_t)1 << f->lmax) - 1;
    for (int b = 0; b < f->lmax; b++)
        for (int d = 0; d < f->dim; d++)
            m |= (uint64_t)(((L->c[d] & mask) >> b) & 1) << (b * f->dim + d);
    return (blk << (f->dim * f->lmax)) | m;
}

typedef struct {
    uint64_t key;
    int64_t idx;
} keyed;

static int cmp_keyed(const void *a, const void *b)
{
    const keyed *x = (const keyed *)a, *y = (const keyed *)b;
    return x->key < y->key ? -1 : x->key > y->key ? 1 : 0;
}

/* sort leaves[n] into brick order; perm (optional) receives the old index of
 * each sorted leaf */
static int sort_leaves(const cipher_forest *f, fleaf *leaves, int64_t n, int64_t *perm)
{
    keyed *k = (keyed *)malloc((size_t)(n > 0 ? n : 1) * sizeof(keyed));
    fleaf *tmp = (fleaf *)malloc((size_t)(n > 0 ? n : 1) * sizeof(fleaf));
    if (!k || !tmp) { free(k); free(tmp); return CIPHER_E_NOMEM; }
    for (int64_t i = 0; i < n; i++) { k[i].key = leaf_key(f, &leaves[i]); k[i].idx = i; }
    qsort(k, (size_t)n, sizeof(keyed), cmp_keyed);
    for (int64_t i = 0; i < n; i++) {
        tmp[i] = leaves[k[i].idx];
        if (perm) perm[i] = k[i].idx;
    }
    memcpy(leaves, tmp, (size_t)n * sizeof(fleaf));
    free(k);
    free(tmp);
    return 0;
}

int cipher_forest_create(int dim, const int32_t *nblocks, int lmin, int lmax, int linit, const int32_t *periodic,
                         const double *size, cipher_forest **out)
{
    *out = NULL;
    if (dim < 1 || dim > 3 || lmin < 0 || lmax < lmin || linit < lmin || linit > lmax || lmax > 20)
        return CIPHER_E_ARG;
    cipher_forest *f = (cipher_forest *)calloc(1, sizeof(cipher_forest));
    if (!f) return CIPHER_E_NOMEM;
    f->dim = dim;
    f->lmin = lmin;
    f->lmax = lmax;
    int64_t fine = 1, nleaf = 1;
    for (int d = 0; d < 3; d++) {
        f->nb[d] = d < dim ? nblocks[d] : 1;
        if (f->nb[d] < 1) { free(f); return CIPHER_E_ARG; }
        f->res[d] = d < dim ? f->nb[d] << lmax : 1;
        f->periodic[d] = d < dim ? (periodic && periodic[d]) : 0;
        f->size[d] = d < dim ? (size ? size[d] : (double)f->res[d]) : 1.0;
        fine *= f->res[d];
        if (d < dim) nleaf *= (int64_t)f->nb[d] << linit;
    }
    /* the finest grid is the resolution of the voxel maps and of cell_global */
    if (fine > ((int64_t)1 << 30)) { free(f); return CIPHER_E_ARG; }
    f->leaf = (fleaf *)malloc((size_t)nleaf * sizeof(fleaf));
    if (!f->leaf) { free(f); return CIPHER_E_NOMEM; }
    const int32_t s = side_of(f, linit);
    int32_t cnt[3] = {1, 1, 1};
    for (int d = 0; d < dim; d++) cnt[d] = f->nb[d] << linit;
    int64_t i = 0;
    for (int32_t z = 0; z < cnt[2]; z++)
        for (int32_t y = 0; y < cnt[1]; y++)
            for (int32_t x = 0; x < cnt[0]; x++) {
                f->leaf[i].level = linit;
                f->leaf[i].c[0] = x * s;
                f->leaf[i].c[1] = dim > 1 ? y * s : 0;
                f->leaf[i].c[2] = dim > 2 ? z * s : 0;
                i++;
            }
    f->n = nleaf;
    int rc = sort_leaves(f, f->leaf, f->n, NULL);
    if (rc) { cipher_forest_destroy(f); return rc; }
    *out = f;
    return 0;
}

void cipher_forest_destroy(cipher_forest *f)
{
    if (!f) return;
    free(f->leaf);
    free(f->src0);
    free(f->nsrc);
    free(f);
}

int64_t cipher_forest_nleaves(const cipher_forest *f) { return f ? f->n : 0; }

int cipher_forest_leaves(const cipher_forest *f, int32_t *level, int32_t *corner)
{
    if (!f) return CIPHER_E_ARG;
    for (int64_t i = 0; i < f->n; i++) {
        if (level) level[i] = f->leaf[i].level;
        if (corner)
            for (int d = 0; d < 3; d++) corner[3 * i + d] = f->leaf[i].c[d];
    }
    return 0;
}

int cipher_forest_resolution(const cipher_forest *f, int32_t *res)
{
    if (!f || !res) return CIPHER_E_ARG;
    for (int d = 0; d < 3; d++) res[d] = f->res[d];
    return 0;
}

/* finest-grid owner map: owner[v] = leaf covering finest cell v */
static int32_t *owner_map(const cipher_forest *f)
{
    const int64_t fine = (int64_t)f->res[0] * f->res[1] * f->res[2];
    int32_t *own = (int32_t *)malloc((size_t)fine * sizeof(int32_t));
    if (!own) return NULL;
    for (int64_t i = 0; i < f->n; i++) {
        const fleaf *L = &f->leaf[i];
        const int32_t s = side_of(f, L->level);
        const int32_t sz = f->dim > 2 ? s : 1, sy = f->dim > 1 ? s : 1;
        for (int32_t z = 0; z < sz; z++)
            for (int32_t y = 0; y < sy; y++) {
                int64_t base = L->c[0] + (int64_t)f->res[0] * ((L->c[1] + y) + (int64_t)f->res[1] * (L->c[2] + z));
                for (int32_t x = 0; x < s; x++) own[base + x] = (int32_t)i;
            }
    }
    return own;
}

/* position across face (d, side) of leaf L on the finest grid, or -1 on a
 * non-periodic boundary */
static int32_t across(const cipher_forest *f, const fleaf *L, int d, int side)
{
    const int32_t s = side_of(f, L->level);
    int32_t p = side ? L->c[d] + s : L->c[d] - 1;
    if (p < 0 || p >= f->res[d]) {
        if (!f->periodic[d]) return -1;
        p = (p + f->res[d]) % f->res[d];
    }
    return p;
}

/* whether a leaf across face (d, side) of L is more than one level finer */
static int face_too_fine(const cipher_forest *f, const int32_t *own, const fleaf *lv, const fleaf *L, int d, int side)
{
    const int32_t p = across(f, L, d, side);
    if (p < 0) return 0;
    const int32_t s = side_of(f, L->level);
    const int e1 = (d + 1) % 3, e2 = (d + 2) % 3;
    const int32_t s1 = e1 < f->dim ? s : 1, s2 = e2 < f->dim ? s : 1;
    for (int32_t b = 0; b < s2; b++)
        for (int32_t a = 0; a < s1; a++) {
            int32_t q[3];
            q[d] = p;
            q[e1] = L->c[e1] + a;
            q[e2] = L->c[e2] + b;
            if (lv[own[q[0] + (int64_t)f->res[0] * (q[1] + (int64_t)f->res[1] * q[2])]].level > L->level + 1)
                return 1;
        }
    return 0;
}

/* the distinct leaves just across face (d, side) of leaf L, ascending
 * (at most `cap`; a balanced forest has at most 2^(dim-1)).  Returns 0 when
 * the face lies on a non-periodic boundary, -1 when there are more than cap. */
static int face_neighbours(const cipher_forest *f, const int32_t *own, const fleaf *L, int d, int side,
                           int32_t *nbr, int *nn, int cap)
{
    const int32_t s = side_of(f, L->level);
    const int32_t p = across(f, L, d, side);
    *nn = 0;
    if (p < 0) return 0;
    int count = 0;
    const int e1 = (d + 1) % 3, e2 = (d + 2) % 3;
    const int32_t s1 = e1 < f->dim ? s : 1, s2 = e2 < f->dim ? s : 1;
    for (int32_t b = 0; b < s2; b++)
        for (int32_t a = 0; a < s1; a++) {
            int32_t q[3];
            q[d] = p;
            q[e1] = L->c[e1] + a;
            q[e2] = L->c[e2] + b;
            const int32_t o = own[q[0] + (int64_t)f->res[0] * (q[1] + (int64_t)f->res[1] * q[2])];
            int k = 0;
            while (k < count && nbr[k] < o) k++;
            if (k < count && nbr[k] == o) continue;
            if (count == cap) return -1;
            for (int j = count; j > k; j--) nbr[j] = nbr[j - 1];
            nbr[k] = o;
            count++;
            *nn = count;
        }
    return 1;
}

/* a leaf of the forest being built, with the old leaves its dofs come
 * from: old leaves [src0, src0 + nsrc) (one leaf, or a coarsened family) */
typedef struct {
    fleaf leaf;
    int64_t src0;
    int32_t nsrc;
} nleaf;

static int sort_nleaves(const cipher_forest *f, nleaf *v, int64_t n)
{
    keyed *k = (keyed *)malloc((size_t)(n > 0 ? n : 1) * sizeof(keyed));
    nleaf *tmp = (nleaf *)malloc((size_t)(n > 0 ? n : 1) * sizeof(nleaf));
    if (!k || !tmp) { free(k); free(tmp); return CIPHER_E_NOMEM; }
    for (int64_t i = 0; i < n; i++) { k[i].key = leaf_key(f, &v[i].leaf); k[i].idx = i; }
    qsort(k, (size_t)n, sizeof(keyed), cmp_keyed);
    for (int64_t i = 0; i < n; i++) tmp[i] = v[k[i].idx];
    memcpy(v, tmp, (size_t)n * sizeof(nleaf));
    free(k);
    free(tmp);
    return 0;
}

/* append the children of L (with L's transfer source) to out */
static void split_into(const cipher_forest *f, const nleaf *L, nleaf *out, int64_t *m)
{
    const int32_t h = side_of(f, L->leaf.level + 1);
    const int nc = 1 << f->dim;
    for (int k = 0; k < nc; k++) {
        nleaf c = *L;
        c.leaf.level = L->leaf.level + 1;
        for (int d = 0; d < f->dim; d++)
            if (k >> d & 1) c.leaf.c[d] += h;
        out[(*m)++] = c;
    }
}

int cipher_forest_adapt(cipher_forest *f, const int8_t *mark, const double *Xold, int ndof, int as_size)
{
    if (!f || !mark || (Xold && (ndof < 1 || as_size < 0 || as_size > ndof))) return CIPHER_E_ARG;
    const int nc = 1 << f->dim;
    const int64_t n0 = f->n;
    /* 1. refine / coarsen by the marks */
    int64_t cap = n0 * nc + nc;
    nleaf *v = (nleaf *)malloc((size_t)cap * sizeof(nleaf));
    if (!v) return CIPHER_E_NOMEM;
    int64_t m = 0;
    for (int64_t i = 0; i < n0;) {
        const fleaf *L = &f->leaf[i];
        int fam = 0;
        if (mark[i] < 0 && L->level > f->lmin && i + nc <= n0) {
            /* a complete family: the next 2^dim leaves share L's parent, all
             * marked coarsen, with the same active set */
            const int32_t ps = side_of(f, L->level - 1);
            int ok = 1;
            for (int d = 0; d < f->dim; d++) if (L->c[d] % ps) ok = 0;
            for (int k = 0; k < nc && ok; k++) {
                const fleaf *S = &f->leaf[i + k];
                if (S->level != L->level || mark[i + k] >= 0) ok = 0;
                for (int d = 0; d < f->dim && ok; d++)
                    if (S->c[d] / ps != L->c[d] / ps) ok = 0;
                if (ok && Xold && as_size > 0 &&
                    memcmp(&Xold[(i + k) * (int64_t)ndof], &Xold[i * (int64_t)ndof], (size_t)as_size * sizeof(double)))
                    ok = 0;
            }
            fam = ok;
        }
        if (fam) {
            v[m].leaf = *L;
            v[m].leaf.level = L->level - 1;
            v[m].src0 = i;
            v[m].nsrc = nc;
            m++;
            i += nc;
        } else {
            nleaf one = {*L, i, 1};
            if (mark[i] > 0 && L->level < f->lmax) split_into(f, &one, v, &m);
            else v[m++] = one;
            i++;
        }
    }
    /* 2. 2:1 balance across faces: a leaf more than one level coarser than a
     * face neighbour splits; repeat until nothing splits */
    cipher_forest cur = *f;
    for (;;) {
        if (sort_nleaves(f, v, m)) { free(v); return CIPHER_E_NOMEM; }
        fleaf *lv = (fleaf *)malloc((size_t)m * sizeof(fleaf));
        if (!lv) { free(v); return CIPHER_E_NOMEM; }
        for (int64_t i = 0; i < m; i++) lv[i] = v[i].leaf;
        cur.leaf = lv;
        cur.n = m;
        int32_t *own = owner_map(&cur);
        if (!own) { free(lv); free(v); return CIPHER_E_NOMEM; }
        char *sp = (char *)calloc((size_t)m, 1);
        int64_t nsplit = 0;
        if (!sp) { free(own); free(lv); free(v); return CIPHER_E_NOMEM; }
        for (int64_t i = 0; i < m; i++) {
            for (int d = 0; d < f->dim && !sp[i]; d++)
                for (int side = 0; side < 2 && !sp[i]; side++)
                    if (face_too_fine(&cur, own, lv, &lv[i], d, side)) { sp[i] = 1; nsplit++; }
        }
        free(own);
        free(lv);
        if (!nsplit) { free(sp); break; }
        nleaf *w = (nleaf *)malloc((size_t)(m + nsplit * (nc - 1)) * sizeof(nleaf));
        if (!w) { free(sp); free(v); return CIPHER_E_NOMEM; }
        int64_t mw = 0;
        for (int64_t i = 0; i < m; i++) {
            if (sp[i]) split_into(f, &v[i], w, &mw);
            else w[mw++] = v[i];
        }
        free(sp);
        free(v);
        v = w;
        m = mw;
    }
    /* 3. install the new leaves and keep the transfer plan */
    fleaf *lv = (fleaf *)malloc((size_t)m * sizeof(fleaf));
    int64_t *s0 = (int64_t *)malloc((size_t)m * sizeof(int64_t));
    int32_t *sn = (int32_t *)malloc((size_t)m * sizeof(int32_t));
    if (!lv || !s0 || !sn) { free(lv); free(s0); free(sn); free(v); return CIPHER_E_NOMEM; }
    for (int64_t i = 0; i < m; i++) {
        lv[i] = v[i].leaf;
        s0[i] = v[i].src0;
        sn[i] = v[i].nsrc;
    }
    free(v);
    free(f->leaf);
    free(f->src0);
    free(f->nsrc);
    f->leaf = lv;
    f->src0 = s0;
    f->nsrc = sn;
    f->n_old = n0;
    f->n = m;
    return 0;
}

int cipher_forest_transfer_plan(const cipher_forest *f, int64_t *src0, int32_t *nsrc)
{
    if (!f || !f->src0) return CIPHER_E_ARG;
    memcpy(src0, f->src0, (size_t)f->n * sizeof(int64_t));
    memcpy(nsrc, f->nsrc, (size_t)f->n * sizeof(int32_t));
    return 0;
}

int cipher_forest_transfer_aos(const cipher_forest *f, const double *Xold, int ndof, double *Xnew)
{
    if (!f || !f->src0 || !Xold || !Xnew || ndof < 1) return CIPHER_E_ARG;
    for (int64_t i = 0; i < f->n; i++) {
        double *o = &Xnew[i * (int64_t)ndof];
        const double *a = &Xold[f->src0[i] * (int64_t)ndof];
        if (f->nsrc[i] == 1) {
            memcpy(o, a, (size_t)ndof * sizeof(double));
            continue;
        }
        /* a coarsened family: the mean of the children, summed in leaf order */
        for (int q = 0; q < ndof; q++) {
            double acc = 0.0;
            for (int k = 0; k < f->nsrc[i]; k++) acc += Xold[(f->src0[i] + k) * (int64_t)ndof + q];
            o[q] = acc / (double)f->nsrc[i];
        }
    }
    return 0;
}

/* the reference's marking (src/cipher.c:1380-1386): refine leaves whose
 * active set holds more than one phase, coarsen the others */
int cipher_forest_mark_active(const cipher_forest *f, const double *X, int ndof, int8_t *mark)
{
    if (!f || !X || !mark || ndof < 1) return CIPHER_E_ARG;
    for (int64_t i = 0; i < f->n; i++) mark[i] = round(X[i * (int64_t)ndof]) > 1 ? 1 : -1;
    return 0;
}

int cipher_forest_mesh(const cipher_forest *f, cipher_mesh **out)
{
    *out = NULL;
    if (!f) return CIPHER_E_ARG;
    if (f->n > 2147483647LL - 1) return CIPHER_E_ARG;
    int32_t *own = owner_map(f);
    if (!own) return CIPHER_E_NOMEM;
    cipher_mesh *m = (cipher_mesh *)calloc(1, sizeof(cipher_mesh));
    const int nc = 1 << (f->dim - 1);
    const int64_t maxf = f->n * f->dim * nc, maxb = f->n * 2 * f->dim;
    if (m) {
        m->cellgeom = (double *)malloc((size_t)f->n * sizeof(double));
        m->cell_global = (int32_t *)malloc((size_t)f->n * sizeof(int32_t));
        m->face_cells = (int32_t *)malloc((size_t)2 * maxf * sizeof(int32_t));
        m->bface_cell = (int32_t *)malloc((size_t)(maxb > 0 ? maxb : 1) * sizeof(int32_t));
        m->bface_label = (int32_t *)malloc((size_t)(maxb > 0 ? maxb : 1) * sizeof(int32_t));
    }
    if (!m || !m->cellgeom || !m->cell_global || !m->face_cells || !m->bface_cell || !m->bface_label) {
        free(own);
        cipher_mesh_free(m);
        return CIPHER_E_NOMEM;
    }
    m->dim = f->dim;
    m->ncells = m->nowned = (int32_t)f->n;
    m->uniform = 0;
    for (int d = 0; d < 3; d++) {
        m->res[d] = f->res[d];
        m->periodic[d] = f->periodic[d] && f->res[d] > 1;
    }
    m->slab_lo = 0;
    m->slab_hi = f->res[f->dim - 1];
    int32_t nbr[64];
    int64_t nf = 0, nbf = 0;
    for (int64_t i = 0; i < f->n; i++) {
        const fleaf *L = &f->leaf[i];
        const int32_t s = side_of(f, L->level);
        /* DMPlexComputeCellGeometryFVM: the volume of the cell; delta = vol^(1/dim) */
        double vol = 1.0;
        for (int d = 0; d < f->dim; d++) vol *= f->size[d] / f->res[d] * s;
        m->cellgeom[i] = pow(vol, 1.0 / f->dim);
        m->cell_global[i] = (int32_t)(L->c[0] + (int64_t)f->res[0] * (L->c[1] + (int64_t)f->res[1] * L->c[2]));
        for (int d = 0; d < f->dim; d++) {
            int nn = 0;
            /* the faces on the upper side of the leaf: this leaf is their L cell */
            const int r = face_neighbours(f, own, L, d, 1, nbr, &nn, 64);
            if (r < 0) { free(own); cipher_mesh_free(m); return CIPHER_E_ARG; }   /* not 2:1 balanced */
            if (r) {
                for (int k = 0; k < nn; k++) {
                    if (nbr[k] == (int32_t)i) continue;     /* a one-leaf periodic direction */
                    m->face_cells[2 * nf] = (int32_t)i;
                    m->face_cells[2 * nf + 1] = nbr[k];
                    nf++;
                }
            }
        }
    }
    /* boundary faces (support 1) of the non-periodic sides, labelled as the
     * reference labels them from the face centroid: 2d+1 low, 2d+2 high */
    for (int64_t i = 0; i < f->n; i++) {
        const fleaf *L = &f->leaf[i];
        const int32_t s = side_of(f, L->level);
        for (int d = 0; d < f->dim; d++) {
            if (f->periodic[d]) continue;
            if (L->c[d] == 0) { m->bface_cell[nbf] = (int32_t)i; m->bface_label[nbf] = 2 * d + 1; nbf++; }
            if (L->c[d] + s == f->res[d]) { m->bface_cell[nbf] = (int32_t)i; m->bface_label[nbf] = 2 * d + 2; nbf++; }
        }
    }
    m->nfaces = (int32_t)nf;
    m->nbfaces = (int32_t)nbf;
    free(own);
    *out = m;
    return 0;
}
