/*
 * oracle_models.c - CPU restatement of CIPHER's thermodynamic model table
 * (src/material.c) and numeric helpers (src/utility.c).
 *
 * TEST INFRASTRUCTURE ONLY: this is the oracle the device kernels are checked
 * against.  Nothing in the product links or calls it.
 *
 * Operation order inside every expression follows the reference so that the
 * IEEE double results agree bit for bit where libm agrees.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"

/* exponentiation by squaring (utility.c:112-124) */
double or_ipow(double base, unsigned e)
{
    double r = 1.0;
    while (e) {
        if (e & 1u) r *= base;
        e >>= 1;
        base *= base;
    }
    return r;
}

/* sum_i c_i T^e_i + l T ln T (utility.c:48-62) */
double or_tseries(double T, const cipher_tseries *s)
{
    double r = 0.0;
    for (int i = 0; i < s->n; i++) {
        if (s->exp[i] > 0) r += s->coeff[i] * or_ipow(T, (unsigned)s->exp[i]);
        else if (s->exp[i] < 0) r += s->coeff[i] / or_ipow(T, (unsigned)(-s->exp[i]));
        else r += s->coeff[i];
    }
    if (fabs(s->logcoeff) > 0.0) r += s->logcoeff * T * log(T);
    return r;
}

/* d/dT of or_tseries (utility.c:67-79) */
double or_tseries_dT(double T, const cipher_tseries *s)
{
    double r = 0.0;
    for (int i = 0; i < s->n; i++) {
        if (s->exp[i] > 0) r += s->exp[i] * s->coeff[i] * or_ipow(T, (unsigned)(s->exp[i] - 1));
        else if (s->exp[i] < 0) r += s->exp[i] * s->coeff[i] / or_ipow(T, (unsigned)(-s->exp[i] + 1));
    }
    if (fabs(s->logcoeff) > 0.0) r += s->logcoeff * (1.0 + log(T));
    return r;
}

/* sorted intersection with positions in A and B (utility.c:168-190) */
int or_set_intersect(const uint16_t *a, int na, const uint16_t *b, int nb,
                     uint16_t *out, uint16_t *ina, uint16_t *inb)
{
    int i = 0, j = 0, n = 0;
    while (i < na && j < nb) {
        if (a[i] == b[j]) { ina[n] = (uint16_t)i; inb[n] = (uint16_t)j; out[n] = a[i]; n++; i++; j++; }
        else if (a[i] < b[j]) i++;
        else j++;
    }
    return n;
}

/* sorted union (utility.c:195-230); returns size, writes at most cap ids */
int or_set_union(const uint16_t *a, int na, const uint16_t *b, int nb, uint16_t *out, int cap)
{
    int i = 0, j = 0, n = 0;
    while (i < na || j < nb) {
        uint16_t v;
        if (j >= nb || (i < na && a[i] < b[j])) v = a[i++];
        else if (i >= na || b[j] < a[i]) v = b[j++];
        else { v = a[i]; i++; j++; }
        if (n < cap) out[n] = v;
        n++;
    }
    return n;
}

/* small dense inverse (utility.c:232-441): closed-form adjugates up to 4x4,
 * Gauss-Jordan above.  src is consumed by the n>4 path. */
void or_invert(double *dst, double *src, int n)
{
    if (n == 1) {
        dst[0] = 1.0 / src[0];
    } else if (n == 2) {
        dst[0] = +src[3];
        dst[2] = -src[2];
        dst[3] = +src[0];
        double det = src[0] * dst[0] + src[1] * dst[2];
        det = 1.0 / det;
        dst[0] *= det; dst[2] *= det; dst[3] *= det;
        dst[1] = dst[2];
    } else if (n == 3) {
        dst[0] = +src[4] * src[8] - src[5] * src[7];
        dst[3] = -src[3] * src[8] + src[5] * src[6];
        dst[4] = +src[0] * src[8] - src[2] * src[6];
        dst[6] = +src[3] * src[7] - src[4] * src[6];
        dst[7] = -src[0] * src[7] + src[1] * src[6];
        dst[8] = +src[0] * src[4] - src[1] * src[3];
        double det = src[0] * dst[0] + src[1] * dst[3] + src[2] * dst[6];
        det = 1.0 / det;
        dst[0] *= det; dst[3] *= det; dst[4] *= det; dst[6] *= det; dst[7] *= det; dst[8] *= det;
        dst[1] = dst[3]; dst[2] = dst[6]; dst[5] = dst[7];
    } else if (n == 4) {
        const double *s = src;
        /* cofactors of the symmetric-fill variant the reference uses: only the
         * lower triangle of the adjugate is formed and mirrored */
        dst[0] = +s[5]*s[10]*s[15] - s[5]*s[11]*s[14] - s[9]*s[6]*s[15] + s[9]*s[7]*s[14] + s[13]*s[6]*s[11] - s[13]*s[7]*s[10];
        dst[4] = -s[4]*s[10]*s[15] + s[4]*s[11]*s[14] + s[8]*s[6]*s[15] - s[8]*s[7]*s[14] - s[12]*s[6]*s[11] + s[12]*s[7]*s[10];
        dst[5] = +s[0]*s[10]*s[15] - s[0]*s[11]*s[14] - s[8]*s[2]*s[15] + s[8]*s[3]*s[14] + s[12]*s[2]*s[11] - s[12]*s[3]*s[10];
        dst[8] = +s[4]*s[9]*s[15] - s[4]*s[11]*s[13] - s[8]*s[5]*s[15] + s[8]*s[7]*s[13] + s[12]*s[5]*s[11] - s[12]*s[7]*s[9];
        dst[9] = -s[0]*s[9]*s[15] + s[0]*s[11]*s[13] + s[8]*s[1]*s[15] - s[8]*s[3]*s[13] - s[12]*s[1]*s[11] + s[12]*s[3]*s[9];
        dst[10] = +s[0]*s[5]*s[15] - s[0]*s[7]*s[13] - s[4]*s[1]*s[15] + s[4]*s[3]*s[13] + s[12]*s[1]*s[7] - s[12]*s[3]*s[5];
        dst[12] = -s[4]*s[9]*s[14] + s[4]*s[10]*s[13] + s[8]*s[5]*s[14] - s[8]*s[6]*s[13] - s[12]*s[5]*s[10] + s[12]*s[6]*s[9];
        dst[13] = +s[0]*s[9]*s[14] - s[0]*s[10]*s[13] - s[8]*s[1]*s[14] + s[8]*s[2]*s[13] + s[12]*s[1]*s[10] - s[12]*s[2]*s[9];
        dst[14] = -s[0]*s[5]*s[14] + s[0]*s[6]*s[13] + s[4]*s[1]*s[14] - s[4]*s[2]*s[13] - s[12]*s[1]*s[6] + s[12]*s[2]*s[5];
        dst[15] = +s[0]*s[5]*s[10] - s[0]*s[6]*s[9] - s[4]*s[1]*s[10] + s[4]*s[2]*s[9] + s[8]*s[1]*s[6] - s[8]*s[2]*s[5];
        double det = +s[0] * dst[0] + s[1] * dst[4] + s[2] * dst[8] + s[3] * dst[12];
        det = 1.0 / det;
        dst[0] *= det; dst[4] *= det; dst[5] *= det; dst[8] *= det; dst[9] *= det;
        dst[10] *= det; dst[12] *= det; dst[13] *= det; dst[14] *= det; dst[15] *= det;
        dst[1] = dst[4]; dst[2] = dst[8]; dst[3] = dst[12];
        dst[6] = dst[9]; dst[7] = dst[13]; dst[11] = dst[14];
    } else {
        memset(dst, 0, (size_t)n * n * sizeof(double));
        for (int i = 0; i < n; i++) dst[i * n + i] = 1.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
                if (i != j) {
                    double ratio = src[j * n + i] / src[i * n + i];
                    for (int k = 0; k < n; k++) src[j * n + k] -= ratio * src[i * n + k];
                    for (int k = 0; k < n; k++) dst[j * n + k] -= ratio * dst[i * n + k];
                }
        for (int i = 0; i < n; i++) {
            double a = src[i * n + i];
            for (int j = 0; j < n; j++) dst[i * n + j] /= a;
        }
    }
}

/* dst = A x (utility.c:456-465) */
void or_matvec(double *dst, const double *A, const double *x, int n)
{
    for (int k = 0; k < n; k++) {
        double acc = 0.0;
        for (int j = 0; j < n; j++) acc += A[k * n + j] * x[j];
        dst[k] = acc;
    }
}

/* phase interpolant h (utility.c:470-535) */
void or_interpolant(int kind, const double *phi, int n, double *h)
{
    if (kind == CIPHER_INTERP_LINEAR) { memcpy(h, phi, (size_t)n * sizeof(double)); return; }
    if (n == 1) { h[0] = 1.0; return; }
    double sum = 0.0;
    for (int g = 0; g < n; g++) {
        h[g] = kind == CIPHER_INTERP_QUADRATIC ? phi[g] * phi[g] : phi[g] * phi[g] * (3.0 - 2.0 * phi[g]);
        sum += h[g];
    }
    for (int g = 0; g < n; g++) h[g] /= sum;
}

/* v <- (dh/dphi)^T v (utility.c:478-557) */
void or_interpolant_dT(int kind, double *v, const double *phi, int n)
{
    if (kind == CIPHER_INTERP_LINEAR) return;
    if (n == 1) { v[0] = 0.0; return; }
    double out[CIPHER_MAXAP];
    double avg = 0.0, sum = 0.0;
    for (int g = 0; g < n; g++) {
        double w = kind == CIPHER_INTERP_QUADRATIC ? phi[g] * phi[g] : phi[g] * phi[g] * (3.0 - 2.0 * phi[g]);
        sum += w;
        avg += w * v[g];
    }
    for (int g = 0; g < n; g++) {
        if (kind == CIPHER_INTERP_QUADRATIC) out[g] = 2.0 * phi[g] * (v[g] - avg / sum) / sum;
        else out[g] = 6.0 * phi[g] * (1.0 - phi[g]) * (v[g] - avg / sum) / sum;
    }
    memcpy(v, out, (size_t)n * sizeof(double));
}

/* Michelot-style projection onto the Gibbs simplex (utility.c:578-603) */
static int cmp_desc(const void *x, const void *y)
{
    double a = *(const double *)x, b = *(const double *)y;
    return b > a ? 1 : (b < a ? -1 : 0);
}
void or_simplex_projection(double *out, const double *in, int n)
{
    double s[CIPHER_MAXAP];
    memcpy(s, in, (size_t)n * sizeof(double));
    qsort(s, (size_t)n, sizeof(double), cmp_desc);
    double sum = 0.0, tmax = 0.0;
    int found = 0;
    for (int i = 0; i < n - 1; i++) {
        sum += s[i];
        tmax = (sum - 1.0) / ((double)(i + 1));
        if (tmax >= s[i + 1]) { found = 1; break; }
    }
    if (!found) tmax = (sum + s[n - 1] - 1.0) / ((double)n);
    for (int i = 0; i < n; i++) out[i] = in[i] - tmax > 0.0 ? in[i] - tmax : 0.0;
}

/* ------------------------------------------------------------------ */
/* model table                                                          */
/* ------------------------------------------------------------------ */

/* raw free energy G(y) per mole (material.c:356-475) */
static double energy_raw(const cipher_material *m, const double *y, double T, int ncp)
{
    double G = 0.0;
    if (m->model == CIPHER_CHEM_NONE) return or_tseries(T, &m->ref);
    if (m->model == CIPHER_CHEM_QUADRATIC) {
        G = or_tseries(T, &m->ref);
        for (int c = 0; c < ncp; c++)
            G += or_tseries(T, &m->unary[c]) * (y[c] - or_tseries(T, &m->quad_ceq[c]))
               + or_tseries(T, &m->quad_binary[c]) * (y[c] - or_tseries(T, &m->quad_ceq[c]))
                                                  * (y[c] - or_tseries(T, &m->quad_ceq[c]));
        return G;
    }
    if (m->model == CIPHER_CHEM_CALPHADDIS) {
        const cipher_rk *bin = m->binary, *ter = m->ternary;
        G = or_tseries(T, &m->ref);
        for (int k = 0; k < ncp; k++) {
            G += or_tseries(T, &m->unary[k]) * y[k] + CIPHER_R_GAS * T * y[k] * log(y[k]);
            for (int j = k + 1; j < ncp; j++, bin++) {
                for (int r = 0; r < bin->n; r++)
                    G += or_tseries(T, &bin->h[r]) * y[k] * y[j] * or_ipow(y[k] - y[j], (unsigned)r);
                for (int i = j + 1; i < ncp; i++, ter++)
                    for (int r = 0; r < ter->n; r++)
                        G += or_tseries(T, &ter->h[r]) * y[k] * y[j] * y[i]
                           * (y[ter->i[r]] + (1.0 - y[k] - y[j] - y[i]) / 3.0);
            }
        }
        return G;
    }
    /* calphad2sl: y = [y_p(ncp) | y_q(ncp)] */
    const double *yp = y, *yq = y + ncp;
    for (int c = 0; c < ncp; c++)
        G += CIPHER_R_GAS * T * (m->p * yp[c] * log(yp[c]) + m->q * yq[c] * log(yq[c]));
    for (int a = 0; a < ncp; a++)
        for (int b = 0; b < ncp; b++)
            G += or_tseries(T, &m->unary[a * ncp + b]) * yp[a] * yq[b];
    const cipher_rk *rk = m->binary;
    for (int i = 0; i < ncp; i++)
        for (int j = i + 1; j < ncp; j++)
            for (int q = 0; q < ncp; q++, rk++)
                for (int r = 0; r < rk->n; r++)
                    G += or_tseries(T, &rk->h[r]) * yp[i] * yp[j] * yq[q] * or_ipow(yp[i] - yp[j], (unsigned)r);
    rk = m->binaryq;
    for (int p = 0; p < ncp; p++)
        for (int i = 0; i < ncp; i++)
            for (int j = i + 1; j < ncp; j++, rk++)
                for (int r = 0; r < rk->n; r++)
                    G += or_tseries(T, &rk->h[r]) * yp[p] * yq[i] * yq[j] * or_ipow(yq[i] - yq[j], (unsigned)r);
    rk = m->ternary;
    for (int i = 0; i < ncp; i++)
        for (int j = i + 1; j < ncp; j++)
            for (int k = j + 1; k < ncp; k++)
                for (int q = 0; q < ncp; q++, rk++)
                    for (int r = 0; r < rk->n; r++)
                        G += or_tseries(T, &rk->h[r]) * yp[i] * yp[j] * yp[k] * yq[q];
    rk = m->ternaryq;
    for (int p = 0; p < ncp; p++)
        for (int i = 0; i < ncp; i++)
            for (int j = i + 1; j < ncp; j++)
                for (int k = j + 1; k < ncp; k++, rk++)
                    for (int r = 0; r < rk->n; r++)
                        G += or_tseries(T, &rk->h[r]) * yq[i] * yq[j] * yq[k] * yp[p];
    return G;
}

/* excess (explicit) potential of every site fraction (material.c:495-635) */
static void explicit_raw(const cipher_material *m, const double *y, double T, int ncp, double *mu)
{
    if (m->model == CIPHER_CHEM_NONE || m->model == CIPHER_CHEM_QUADRATIC) {
        memset(mu, 0, (size_t)ncp * sizeof(double));
        return;
    }
    if (m->model == CIPHER_CHEM_CALPHADDIS) {
        for (int i = 0; i < ncp; i++) mu[i] = or_tseries(T, &m->unary[i]);
        const cipher_rk *bin = m->binary;
        for (int i = 0; i < ncp; i++)
            for (int j = i + 1; j < ncp; j++, bin++)
                for (int r = 0; r < bin->n; r++) {
                    double a = or_tseries(T, &bin->h[r]);
                    double b = or_ipow(y[i] - y[j], (unsigned)r);
                    double c = r == 0 ? 0.0 : ((double)r) * or_ipow(y[i] - y[j], (unsigned)(r - 1));
                    mu[i] += a * y[j] * (b + c * y[i]);
                    mu[j] += a * y[i] * (b - c * y[j]);
                }
        const cipher_rk *ter = m->ternary;
        for (int i = 0; i < ncp; i++)
            for (int j = i + 1; j < ncp; j++)
                for (int k = j + 1; k < ncp; k++, ter++)
                    for (int r = 0; r < ter->n; r++) {
                        double a = or_tseries(T, &ter->h[r]);
                        double b = y[ter->i[r]] + (1.0 - y[k] - y[j] - y[i]) / 3.0;
                        mu[i] += a * y[j] * y[k] * (b - y[i] / 3.0);
                        mu[j] += a * y[k] * y[i] * (b - y[j] / 3.0);
                        mu[k] += a * y[i] * y[j] * (b - y[k] / 3.0);
                        mu[ter->i[r]] += a * y[i] * y[j] * y[k];
                    }
        return;
    }
    const double *yp = y, *yq = y + ncp;
    double *mp = mu, *mq = mu + ncp;
    memset(mu, 0, 2 * (size_t)ncp * sizeof(double));
    for (int a = 0; a < ncp; a++)
        for (int b = 0; b < ncp; b++) {
            double w = or_tseries(T, &m->unary[a * ncp + b]);
            mp[a] += w * yq[b];
            mq[b] += w * yp[a];
        }
    const cipher_rk *rk = m->binary;
    for (int i = 0; i < ncp; i++)
        for (int j = i + 1; j < ncp; j++)
            for (int q = 0; q < ncp; q++, rk++)
                for (int r = 0; r < rk->n; r++) {
                    double a = or_tseries(T, &rk->h[r]);
                    double b = or_ipow(yp[i] - yp[j], (unsigned)r);
                    double c = r == 0 ? 0.0 : ((double)r) * or_ipow(yp[i] - yp[j], (unsigned)(r - 1));
                    mp[i] += a * yp[j] * yq[q] * (b + c * yp[i]);
                    mp[j] += a * yp[i] * yq[q] * (b - c * yp[j]);
                    mq[q] += a * yp[i] * b * yp[j];
                }
    rk = m->binaryq;
    for (int p = 0; p < ncp; p++)
        for (int i = 0; i < ncp; i++)
            for (int j = i + 1; j < ncp; j++, rk++)
                for (int r = 0; r < rk->n; r++) {
                    double a = or_tseries(T, &rk->h[r]);
                    double b = or_ipow(yq[i] - yq[j], (unsigned)r);
                    double c = r == 0 ? 0.0 : ((double)r) * or_ipow(yq[i] - yq[j], (unsigned)(r - 1));
                    mq[i] += a * yq[j] * yp[p] * (b + c * yq[i]);
                    mq[j] += a * yq[i] * yp[p] * (b - c * yq[j]);
                    mp[p] += a * yq[i] * b * yq[j];
                }
    rk = m->ternary;
    for (int i = 0; i < ncp; i++)
        for (int j = i + 1; j < ncp; j++)
            for (int k = j + 1; k < ncp; k++)
                for (int q = 0; q < ncp; q++, rk++)
                    for (int r = 0; r < rk->n; r++) {
                        double a = or_tseries(T, &rk->h[r]);
                        mp[i] += a * yp[j] * yp[k] * yq[q];
                        mp[j] += a * yp[k] * yp[i] * yq[q];
                        mp[k] += a * yp[i] * yp[j] * yq[q];
                        mq[q] += a * yp[i] * yp[j] * yp[k];
                    }
    rk = m->ternaryq;
    for (int p = 0; p < ncp; p++)
        for (int i = 0; i < ncp; i++)
            for (int j = i + 1; j < ncp; j++)
                for (int k = j + 1; k < ncp; k++, rk++)
                    for (int r = 0; r < rk->n; r++) {
                        double a = or_tseries(T, &rk->h[r]);
                        mq[i] += a * yq[j] * yq[k] * yp[p];
                        mq[j] += a * yq[k] * yq[i] * yp[p];
                        mq[k] += a * yq[i] * yq[j] * yp[p];
                        mp[p] += a * yq[i] * yq[j] * yq[k];
                    }
}

/* ideal (implicit) potential of every site fraction (material.c:655-696) */
static void implicit_raw(const cipher_material *m, const double *y, double T, int ncp, double *mu)
{
    if (m->model == CIPHER_CHEM_NONE) { memset(mu, 0, (size_t)ncp * sizeof(double)); return; }
    if (m->model == CIPHER_CHEM_QUADRATIC) {
        for (int c = 0; c < ncp; c++)
            mu[c] = or_tseries(T, &m->unary[c])
                  + 2.0 * or_tseries(T, &m->quad_binary[c]) * (y[c] - or_tseries(T, &m->quad_ceq[c]));
        return;
    }
    if (m->model == CIPHER_CHEM_CALPHADDIS) {
        for (int c = 0; c < ncp; c++) mu[c] = CIPHER_R_GAS * T * log(y[c]);
        return;
    }
    for (int c = 0; c < ncp; c++) {
        mu[c] = CIPHER_R_GAS * T * m->p * log(y[c]);
        mu[ncp + c] = CIPHER_R_GAS * T * m->q * log(y[ncp + c]);
    }
}

/* site fractions from the implicit site potential (material.c:732-807) */
static void sitefrac_raw(const cipher_material *m, const double *pot, double T, int ncp, double *y)
{
    int nd = ncp - 1;
    if (m->model == CIPHER_CHEM_NONE) {
        memset(y, 0, (size_t)ncp * sizeof(double));
        y[ncp - 1] = 1.0;
        return;
    }
    if (m->model == CIPHER_CHEM_CALPHADDIS) {
        double RT = CIPHER_R_GAS * T, sum = 1.0;
        for (int c = 0; c < nd; c++) { y[c] = exp(pot[c] / RT); sum += y[c]; }
        y[nd] = 1.0;
        for (int c = 0; c < nd; c++) { y[c] /= sum; y[nd] -= y[c]; }
        return;
    }
    if (m->model == CIPHER_CHEM_CALPHAD2SL) {
        double RT = CIPHER_R_GAS * T, sp = 1.0, sq = 1.0;
        double *yp = y, *yq = y + ncp;
        const double *pp = pot, *pq = pot + nd;
        for (int c = 0; c < nd; c++) {
            yp[c] = exp(pp[c] / m->p / RT); sp += yp[c];
            yq[c] = exp(pq[c] / m->q / RT); sq += yq[c];
        }
        yp[nd] = 1.0; yq[nd] = 1.0;
        for (int c = 0; c < nd; c++) {
            yp[c] /= sp; yp[nd] -= yp[c];
            yq[c] /= sq; yq[nd] -= yq[c];
        }
        return;
    }
    /* quadratic: one linear solve */
    double delta[CIPHER_MAXCP], ceq[CIPHER_MAXCP], un[CIPHER_MAXCP], bi[CIPHER_MAXCP];
    double mat[CIPHER_MAXCP * CIPHER_MAXCP], inv[CIPHER_MAXCP * CIPHER_MAXCP];
    for (int c = 0; c < ncp; c++) {
        ceq[c] = or_tseries(T, &m->quad_ceq[c]);
        un[c] = or_tseries(T, &m->unary[c]);
        bi[c] = or_tseries(T, &m->quad_binary[c]);
    }
    memset(mat, 0, sizeof(mat));
    memset(inv, 0, sizeof(inv));
    for (int j = 0; j < nd; j++) {
        delta[j] = 0.5 * pot[j] + bi[nd] - 0.5 * (un[j] - un[nd]) + (bi[j] * ceq[j] - bi[nd] * ceq[nd]);
        mat[j * nd + j] += bi[j];
        for (int i = 0; i < nd; i++) mat[j * nd + i] += bi[nd];
    }
    or_invert(inv, mat, nd);
    or_matvec(y, inv, delta, nd);
    y[nd] = 1.0;
    for (int c = 0; c < nd; c++) y[nd] -= y[c];
}

/* d y / d(pot), d y / d(ex), d y / dT per site (material.c:827-990) */
static void tangent_raw(const cipher_material *m, const double *y, const double *pot, double T, int ncp,
                        double *tpot, double *tex, double *tT)
{
    int nd = ncp - 1, nd2 = nd * nd;
    if (m->model == CIPHER_CHEM_NONE) {
        memset(tpot, 0, (size_t)nd2 * sizeof(double));
        memset(tex, 0, (size_t)nd2 * sizeof(double));
        memset(tT, 0, (size_t)nd * sizeof(double));
        return;
    }
    if (m->model == CIPHER_CHEM_CALPHADDIS) {
        double RT = CIPHER_R_GAS * T, t[CIPHER_MAXCP * CIPHER_MAXCP];
        memset(t, 0, sizeof(t));
        for (int j = 0; j < nd; j++) {
            t[j * nd + j] += y[j] / RT;
            for (int i = 0; i < nd; i++) t[j * nd + i] -= y[j] * y[i] / RT;
        }
        for (int c = 0; c < nd2; c++) { tpot[c] = t[c]; tex[c] = -t[c]; }
        memset(tT, 0, (size_t)nd * sizeof(double));
        for (int j = 0; j < nd; j++)
            for (int i = 0; i < nd; i++) tT[j] -= t[j * nd + i] * pot[i] / T;
        return;
    }
    if (m->model == CIPHER_CHEM_CALPHAD2SL) {
        double RT = CIPHER_R_GAS * T, tp[CIPHER_MAXCP * CIPHER_MAXCP], tq[CIPHER_MAXCP * CIPHER_MAXCP];
        const double *yp = y, *yq = y + ncp, *pp = pot, *pq = pot + nd;
        memset(tp, 0, sizeof(tp));
        memset(tq, 0, sizeof(tq));
        for (int j = 0; j < nd; j++) {
            tp[j * nd + j] += yp[j] / m->p / RT;
            tq[j * nd + j] += yq[j] / m->q / RT;
            for (int i = 0; i < nd; i++) {
                tp[j * nd + i] -= yp[j] * yp[i] / m->p / RT;
                tq[j * nd + i] -= yq[j] * yq[i] / m->q / RT;
            }
        }
        for (int c = 0; c < nd2; c++) {
            tpot[c] = tp[c]; tpot[nd2 + c] = tq[c];
            tex[c] = -tp[c]; tex[nd2 + c] = -tq[c];
        }
        memset(tT, 0, 2 * (size_t)nd * sizeof(double));
        for (int j = 0; j < nd; j++)
            for (int i = 0; i < nd; i++) {
                tT[j] -= tp[j * nd + i] * pp[i] / T;
                tT[nd + j] -= tq[j * nd + i] * pq[i] / T;
            }
        return;
    }
    /* quadratic */
    double delta[CIPHER_MAXCP], ceqT[CIPHER_MAXCP], unT[CIPHER_MAXCP], biT[CIPHER_MAXCP];
    double ceq[CIPHER_MAXCP], bi[CIPHER_MAXCP];
    double mat[CIPHER_MAXCP * CIPHER_MAXCP], inv[CIPHER_MAXCP * CIPHER_MAXCP];
    for (int c = 0; c < ncp; c++) {
        ceqT[c] = or_tseries_dT(T, &m->quad_ceq[c]);
        unT[c] = or_tseries_dT(T, &m->unary[c]);
        biT[c] = or_tseries_dT(T, &m->quad_binary[c]);
        ceq[c] = or_tseries(T, &m->quad_ceq[c]);
        bi[c] = or_tseries(T, &m->quad_binary[c]);
    }
    memset(mat, 0, sizeof(mat));
    memset(inv, 0, sizeof(inv));
    for (int j = 0; j < nd; j++) {
        mat[j * nd + j] += bi[j];
        for (int i = 0; i < nd; i++) mat[j * nd + i] += bi[nd];
    }
    or_invert(inv, mat, nd);
    memcpy(tpot, inv, (size_t)nd2 * sizeof(double));
    for (int c = 0; c < nd2; c++) tpot[c] *= 0.5;
    memset(tex, 0, (size_t)nd2 * sizeof(double));
    memset(tT, 0, (size_t)nd * sizeof(double));
    for (int j = 0; j < nd; j++)
        delta[j] = biT[nd] - 0.5 * (unT[j] - unT[nd])
                 + (biT[j] * ceq[j] + bi[j] * ceqT[j] - biT[nd] * ceq[nd] - bi[nd] * ceqT[nd]);
    or_matvec(tT, inv, delta, nd);
}

/* lattice-fixed component mobility (material.c:1023-1110) */
static void mobility_raw(const cipher_material *m, const double *y, double T, int ncp, double *M)
{
    if (m->model == CIPHER_CHEM_NONE) { memset(M, 0, (size_t)ncp * sizeof(double)); return; }
    for (int k = 0; k < ncp; k++) {
        const cipher_mobility *mob = &m->mobilityc[k];
        const cipher_rk *bin = mob->binary;
        double mig = 0.0;
        for (int j = 0; j < ncp; j++) {
            mig += y[j] * or_tseries(T, &mob->unary[j]);
            for (int i = j + 1; i < ncp; i++, bin++)
                for (int r = 0; r < bin->n; r++)
                    mig += y[j] * y[i] * or_tseries(T, &bin->h[r]) * or_ipow(y[j] - y[i], (unsigned)r);
        }
        M[k] = y[k] * mob->m0 / CIPHER_R_GAS / T * exp(mig / CIPHER_R_GAS / T);
    }
}

/* ---- scaled per-phase wrappers (material.c:480-490, 640-650, 701-727, 812-822, 995-1018, 1115-1120) ---- */

const cipher_material *or_material(const cipher_problem *p, int phase)
{
    return &p->material[p->phasematerialmapping[phase]];
}

double or_chemenergy(const cipher_problem *p, int phase, const double *y, const double *mu, double T)
{
    const cipher_material *m = or_material(p, phase);
    double G = energy_raw(m, y, T, p->ncp) / m->molarvolume;
    for (int s = 0; s < m->nsites; s++)
        for (int c = 0; c < p->ndp; c++) G -= mu[c] * m->stoichiometry[s] * y[s * p->ncp + c];
    return G;
}

void or_sitepot_explicit(const cipher_problem *p, int phase, const double *y, double T, double *out)
{
    const cipher_material *m = or_material(p, phase);
    double full[2 * CIPHER_MAXCP];
    explicit_raw(m, y, T, p->ncp, full);
    for (int s = 0; s < m->nsites; s++)
        for (int c = 0; c < p->ndp; c++)
            out[s * p->ndp + c] = (full[s * p->ncp + c] - full[s * p->ncp + p->ndp]) / m->molarvolume;
}

void or_sitepot_total(const cipher_problem *p, int phase, const double *y, double T, double *out)
{
    const cipher_material *m = or_material(p, phase);
    double full[2 * CIPHER_MAXCP], im[2 * CIPHER_MAXCP], ex[2 * CIPHER_MAXCP];
    implicit_raw(m, y, T, p->ncp, full);
    for (int s = 0; s < m->nsites; s++)
        for (int c = 0; c < p->ndp; c++)
            im[s * p->ndp + c] = (full[s * p->ncp + c] - full[s * p->ncp + p->ndp]) / m->molarvolume;
    or_sitepot_explicit(p, phase, y, T, ex);
    for (int s = 0; s < m->nsites; s++)
        for (int c = 0; c < p->ndp; c++) out[s * p->ndp + c] = im[s * p->ndp + c] + ex[s * p->ndp + c];
}

void or_sitefrac(const cipher_problem *p, int phase, const double *pot, double T, double *y)
{
    const cipher_material *m = or_material(p, phase);
    double scaled[2 * CIPHER_MAXCP];
    for (int s = 0; s < m->nsites; s++)
        for (int c = 0; c < p->ndp; c++) scaled[s * p->ndp + c] = m->molarvolume * pot[s * p->ndp + c];
    sitefrac_raw(m, scaled, T, p->ncp, y);
}

void or_sitefrac_tangent(const cipher_problem *p, int phase, const double *y, const double *pot, double T,
                         double *tpot, double *tex, double *tT)
{
    const cipher_material *m = or_material(p, phase);
    tangent_raw(m, y, pot, T, p->ncp, tpot, tex, tT);
    int nd = p->ndp;
    for (int c = 0; c < m->nsites * nd * nd; c++) tpot[c] *= m->molarvolume;
    for (int c = 0; c < m->nsites * nd * nd; c++) tex[c] *= m->molarvolume;
    for (int c = 0; c < m->nsites * nd; c++) tT[c] *= m->molarvolume;
}

void or_mobility(const cipher_problem *p, int phase, const double *y, double T, double *M)
{
    const cipher_material *m = or_material(p, phase);
    mobility_raw(m, y, T, p->ncp, M);
    for (int c = 0; c < p->ncp; c++) M[c] *= m->molarvolume;
}

/* the raw model functions for the nucleation restatement */
double or_energy_raw(const cipher_material *m, const double *y, double T, int ncp) { return energy_raw(m, y, T, ncp); }
void or_mobility_raw(const cipher_material *m, const double *y, double T, int ncp, double *M) { mobility_raw(m, y, T, ncp, M); }
