/*
 * models.cuh - thermodynamic model table of CIPHER on the device
 * (src/material.c: none, quadratic, calphaddis = one-sublattice CEF with
 * Redlich-Kister excess, calphad2sl = two-sublattice CEF p:q) and the small
 * dense helpers it needs (src/utility.c).
 *
 * Materials are the host structs of include/cipher_problem.h copied to
 * device memory unchanged; the RK tables are walked in the reference's
 * pair/triple enumeration order.  All arithmetic is FP64 in the reference's
 * operation order (this header is only used by units compiled with
 * --fmad=false), so results differ from the reference only where CUDA's exp
 * and log differ from the host libm in the last bit.
 */
#pragma once
#include <cstdint>
#include "device_common.cuh"

namespace cipher {

__device__ __forceinline__ const cipher_material &material_of(const ChemTables &t, int phase)
{
    return t.mat[t.pmm[phase]];
}

__device__ inline double tseries_dT(double T, const cipher_tseries &s)
{
    double r = 0.0;
    for (int i = 0; i < s.n; i++) {
        int e = s.exp[i];
        if (e > 0) r += e * s.coeff[i] * ipow(T, (unsigned)(e - 1));
        else if (e < 0) r += e * s.coeff[i] / ipow(T, (unsigned)(-e + 1));
    }
    if (fabs(s.logcoeff) > 0.0) r += s.logcoeff * (1.0 + log(T));
    return r;
}

/* the evaluated tables serve the CALPHAD models only, whose bodies take no
 * T-derivative; present so that the quadratic branches compile */
__device__ __forceinline__ double tseries_dT(double, const TsV &) { return 0.0; }

/* closed-form inverses for the symmetric matrices of the path (n <= 4,
 * src/utility.c:232-405; only the lower-triangle cofactors are formed) */
__device__ __forceinline__ void invert_small(double *dst, const double *src, int n)
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
        const double *s = src;
        dst[0] = +s[4] * s[8] - s[5] * s[7];
        dst[3] = -s[3] * s[8] + s[5] * s[6];
        dst[4] = +s[0] * s[8] - s[2] * s[6];
        dst[6] = +s[3] * s[7] - s[4] * s[6];
        dst[7] = -s[0] * s[7] + s[1] * s[6];
        dst[8] = +s[0] * s[4] - s[1] * s[3];
        double det = s[0] * dst[0] + s[1] * dst[3] + s[2] * dst[6];
        det = 1.0 / det;
        dst[0] *= det; dst[3] *= det; dst[4] *= det; dst[6] *= det; dst[7] *= det; dst[8] *= det;
        dst[1] = dst[3]; dst[2] = dst[6]; dst[5] = dst[7];
    } else {
        const double *s = src;
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
    }
}

__device__ __forceinline__ void matvec(double *dst, const double *A, const double *x, int n)
{
    for (int k = 0; k < n; k++) {
        double acc = 0.0;
        for (int j = 0; j < n; j++) acc += A[k * n + j] * x[j];
        dst[k] = acc;
    }
}

/* v[i] for a component index i read from a table: with a compile-time
 * count NC a select over the components, so v can stay in registers */
template <int NC>
__device__ __forceinline__ double pick(const double *v, int i)
{
    if constexpr (NC > 0) {
        double r = v[0];
#pragma unroll
        for (int k = 1; k < NC; k++) r = i == k ? v[k] : r;
        return r;
    } else {
        return v[i];
    }
}

template <int NC>
__device__ __forceinline__ void add_at(double *v, int i, double x)
{
    if constexpr (NC > 0) {
#pragma unroll
        for (int k = 0; k < NC; k++)
            if (i == k) v[k] += x;
    } else {
        v[i] += x;
    }
}

/* sublattices of a chemical model (cipher_problem_finalize) */
__host__ __device__ constexpr int model_nsites(int model)
{
    return model == CIPHER_CHEM_NONE ? 0 : model == CIPHER_CHEM_CALPHAD2SL ? 2 : 1;
}

/* ---------------- raw model functions (per mole) ---------------- */

template <int NC, int MODEL, typename Mat>
static __device__ __forceinline__ double energy_body(const Mat &m, const double *y, double T, int ncp_rt)
{
    const int ncp = NC > 0 ? NC : ncp_rt;
    const int model = MODEL >= 0 ? MODEL : m.model;

    if (model == CIPHER_CHEM_NONE) return tseries(T, m.ref);
    if (model == CIPHER_CHEM_QUADRATIC) {
        double G = tseries(T, m.ref);
        for (int c = 0; c < ncp; c++)
            G += tseries(T, m.unary[c]) * (y[c] - tseries(T, m.quad_ceq[c]))
               + tseries(T, m.quad_binary[c]) * (y[c] - tseries(T, m.quad_ceq[c])) * (y[c] - tseries(T, m.quad_ceq[c]));
        return G;
    }
    if (model == CIPHER_CHEM_CALPHADDIS) {
        const auto *bin = m.binary;
        const auto *ter = m.ternary;
        double G = tseries(T, m.ref);
        for (int k = 0; k < ncp; k++) {
            G += tseries(T, m.unary[k]) * y[k] + CIPHER_R_GAS * T * y[k] * log(y[k]);
            for (int j = k + 1; j < ncp; j++, bin++) {
                for (int r = 0; r < bin->n; r++)
                    G += tseries(T, bin->h[r]) * y[k] * y[j] * ipow(y[k] - y[j], (unsigned)r);
                for (int i = j + 1; i < ncp; i++, ter++)
                    for (int r = 0; r < ter->n; r++)
                        G += tseries(T, ter->h[r]) * y[k] * y[j] * y[i] * (pick<NC>(y, ter->i[r]) + (1.0 - y[k] - y[j] - y[i]) / 3.0);
            }
        }
        return G;
    }
    const double *yp = y, *yq = y + ncp;
    double G = 0.0;
    for (int c = 0; c < ncp; c++) G += CIPHER_R_GAS * T * (m.p * yp[c] * log(yp[c]) + m.q * yq[c] * log(yq[c]));
    for (int a = 0; a < ncp; a++) {
        for (int b = 0; b < ncp; b++) G += tseries(T, m.unary[a * ncp + b]) * yp[a] * yq[b];
    }
    const auto *rk = m.binary;
    for (int i = 0; i < ncp; i++) {
        for (int j = i + 1; j < ncp; j++) {
            for (int q = 0; q < ncp; q++, rk++)
                for (int r = 0; r < rk->n; r++)
                    G += tseries(T, rk->h[r]) * yp[i] * yp[j] * yq[q] * ipow(yp[i] - yp[j], (unsigned)r);
        }
    }
    rk = m.binaryq;
    for (int p = 0; p < ncp; p++) {
        for (int i = 0; i < ncp; i++) {
            for (int j = i + 1; j < ncp; j++, rk++)
                for (int r = 0; r < rk->n; r++)
                    G += tseries(T, rk->h[r]) * yp[p] * yq[i] * yq[j] * ipow(yq[i] - yq[j], (unsigned)r);
        }
    }
    rk = m.ternary;
    for (int i = 0; i < ncp; i++) {
        for (int j = i + 1; j < ncp; j++) {
            for (int k = j + 1; k < ncp; k++) {
                for (int q = 0; q < ncp; q++, rk++)
                    for (int r = 0; r < rk->n; r++) G += tseries(T, rk->h[r]) * yp[i] * yp[j] * yp[k] * yq[q];
            }
        }
    }
    rk = m.ternaryq;
    for (int p = 0; p < ncp; p++) {
        for (int i = 0; i < ncp; i++) {
            for (int j = i + 1; j < ncp; j++) {
                for (int k = j + 1; k < ncp; k++, rk++)
                    for (int r = 0; r < rk->n; r++) G += tseries(T, rk->h[r]) * yq[i] * yq[j] * yq[k] * yp[p];
            }
        }
    }
    return G;
}

static __device__ __noinline__ double energy_raw(const cipher_material &m, const double *y, double T, int ncp)
{
    return energy_body<0, -1>(m, y, T, ncp);
}

template <int NC, int MODEL, typename Mat>
static __device__ __forceinline__ void explicit_body(const Mat &m, const double *y, double T, int ncp_rt, double *mu)
{
    const int ncp = NC > 0 ? NC : ncp_rt;
    const int model = MODEL >= 0 ? MODEL : m.model;

    if (model == CIPHER_CHEM_NONE || model == CIPHER_CHEM_QUADRATIC) {
        for (int c = 0; c < ncp; c++) mu[c] = 0.0;
        return;
    }
    if (model == CIPHER_CHEM_CALPHADDIS) {
        for (int i = 0; i < ncp; i++) mu[i] = tseries(T, m.unary[i]);
        const auto *bin = m.binary;
        for (int i = 0; i < ncp; i++) {
            for (int j = i + 1; j < ncp; j++, bin++)
                for (int r = 0; r < bin->n; r++) {
                    double a = tseries(T, bin->h[r]);
                    double b = ipow(y[i] - y[j], (unsigned)r);
                    double c = r == 0 ? 0.0 : ((double)r) * ipow(y[i] - y[j], (unsigned)(r - 1));
                    mu[i] += a * y[j] * (b + c * y[i]);
                    mu[j] += a * y[i] * (b - c * y[j]);
                }
        }
        const auto *ter = m.ternary;
        for (int i = 0; i < ncp; i++) {
            for (int j = i + 1; j < ncp; j++) {
                for (int k = j + 1; k < ncp; k++, ter++)
                    for (int r = 0; r < ter->n; r++) {
                        double a = tseries(T, ter->h[r]);
                        double b = pick<NC>(y, ter->i[r]) + (1.0 - y[k] - y[j] - y[i]) / 3.0;
                        mu[i] += a * y[j] * y[k] * (b - y[i] / 3.0);
                        mu[j] += a * y[k] * y[i] * (b - y[j] / 3.0);
                        mu[k] += a * y[i] * y[j] * (b - y[k] / 3.0);
                        add_at<NC>(mu, ter->i[r], a * y[i] * y[j] * y[k]);
                    }
            }
        }
        return;
    }
    const double *yp = y, *yq = y + ncp;
    double *mp = mu, *mq = mu + ncp;
    for (int c = 0; c < 2 * ncp; c++) mu[c] = 0.0;
    for (int a = 0; a < ncp; a++) {
        for (int b = 0; b < ncp; b++) {
            double w = tseries(T, m.unary[a * ncp + b]);
            mp[a] += w * yq[b];
            mq[b] += w * yp[a];
        }
    }
    const auto *rk = m.binary;
    for (int i = 0; i < ncp; i++) {
        for (int j = i + 1; j < ncp; j++) {
            for (int q = 0; q < ncp; q++, rk++)
                for (int r = 0; r < rk->n; r++) {
                    double a = tseries(T, rk->h[r]);
                    double b = ipow(yp[i] - yp[j], (unsigned)r);
                    double c = r == 0 ? 0.0 : ((double)r) * ipow(yp[i] - yp[j], (unsigned)(r - 1));
                    mp[i] += a * yp[j] * yq[q] * (b + c * yp[i]);
                    mp[j] += a * yp[i] * yq[q] * (b - c * yp[j]);
                    mq[q] += a * yp[i] * b * yp[j];
                }
        }
    }
    rk = m.binaryq;
    for (int p = 0; p < ncp; p++) {
        for (int i = 0; i < ncp; i++) {
            for (int j = i + 1; j < ncp; j++, rk++)
                for (int r = 0; r < rk->n; r++) {
                    double a = tseries(T, rk->h[r]);
                    double b = ipow(yq[i] - yq[j], (unsigned)r);
                    double c = r == 0 ? 0.0 : ((double)r) * ipow(yq[i] - yq[j], (unsigned)(r - 1));
                    mq[i] += a * yq[j] * yp[p] * (b + c * yq[i]);
                    mq[j] += a * yq[i] * yp[p] * (b - c * yq[j]);
                    mp[p] += a * yq[i] * b * yq[j];
                }
        }
    }
    rk = m.ternary;
    for (int i = 0; i < ncp; i++) {
        for (int j = i + 1; j < ncp; j++) {
            for (int k = j + 1; k < ncp; k++) {
                for (int q = 0; q < ncp; q++, rk++)
                    for (int r = 0; r < rk->n; r++) {
                        double a = tseries(T, rk->h[r]);
                        mp[i] += a * yp[j] * yp[k] * yq[q];
                        mp[j] += a * yp[k] * yp[i] * yq[q];
                        mp[k] += a * yp[i] * yp[j] * yq[q];
                        mq[q] += a * yp[i] * yp[j] * yp[k];
                    }
            }
        }
    }
    rk = m.ternaryq;
    for (int p = 0; p < ncp; p++) {
        for (int i = 0; i < ncp; i++) {
            for (int j = i + 1; j < ncp; j++) {
                for (int k = j + 1; k < ncp; k++, rk++)
                    for (int r = 0; r < rk->n; r++) {
                        double a = tseries(T, rk->h[r]);
                        mq[i] += a * yq[j] * yq[k] * yp[p];
                        mq[j] += a * yq[k] * yq[i] * yp[p];
                        mq[k] += a * yq[i] * yq[j] * yp[p];
                        mp[p] += a * yq[i] * yq[j] * yq[k];
                    }
            }
        }
    }
}

static __device__ __noinline__ void explicit_raw(const cipher_material &m, const double *y, double T, int ncp, double *mu)
{
    explicit_body<0, -1>(m, y, T, ncp, mu);
}

template <int NC, int MODEL, typename Mat>
static __device__ __forceinline__ void implicit_body(const Mat &m, const double *y, double T, int ncp_rt, double *mu)
{
    const int ncp = NC > 0 ? NC : ncp_rt;
    const int model = MODEL >= 0 ? MODEL : m.model;

    if (model == CIPHER_CHEM_NONE) {
        for (int c = 0; c < ncp; c++) mu[c] = 0.0;
    } else if (model == CIPHER_CHEM_QUADRATIC) {
        for (int c = 0; c < ncp; c++)
            mu[c] = tseries(T, m.unary[c]) + 2.0 * tseries(T, m.quad_binary[c]) * (y[c] - tseries(T, m.quad_ceq[c]));
    } else if (model == CIPHER_CHEM_CALPHADDIS) {
        for (int c = 0; c < ncp; c++) mu[c] = CIPHER_R_GAS * T * log(y[c]);
    } else {
        for (int c = 0; c < ncp; c++) {
            mu[c] = CIPHER_R_GAS * T * m.p * log(y[c]);
            mu[ncp + c] = CIPHER_R_GAS * T * m.q * log(y[ncp + c]);
        }
    }
}

static __device__ __noinline__ void implicit_raw(const cipher_material &m, const double *y, double T, int ncp, double *mu)
{
    implicit_body<0, -1>(m, y, T, ncp, mu);
}

template <int NC, int MODEL, typename Mat>
static __device__ __forceinline__ void sitefrac_body(const Mat &m, const double *pot, double T, int ncp_rt, double *y)
{
    const int ncp = NC > 0 ? NC : ncp_rt;
    const int model = MODEL >= 0 ? MODEL : m.model;

    const int nd = ncp - 1;
    if (model == CIPHER_CHEM_NONE) {
        for (int c = 0; c < ncp; c++) y[c] = 0.0;
        y[ncp - 1] = 1.0;
    } else if (model == CIPHER_CHEM_CALPHADDIS) {
        double RT = CIPHER_R_GAS * T, sum = 1.0;
        for (int c = 0; c < nd; c++) { y[c] = exp(pot[c] / RT); sum += y[c]; }
        y[nd] = 1.0;
        for (int c = 0; c < nd; c++) { y[c] /= sum; y[nd] -= y[c]; }
    } else if (model == CIPHER_CHEM_CALPHAD2SL) {
        double RT = CIPHER_R_GAS * T, sp = 1.0, sq = 1.0;
        double *yp = y, *yq = y + ncp;
        const double *pp = pot, *pq = pot + nd;
        for (int c = 0; c < nd; c++) {
            yp[c] = exp(pp[c] / m.p / RT); sp += yp[c];
            yq[c] = exp(pq[c] / m.q / RT); sq += yq[c];
        }
        yp[nd] = 1.0; yq[nd] = 1.0;
        for (int c = 0; c < nd; c++) {
            yp[c] /= sp; yp[nd] -= yp[c];
            yq[c] /= sq; yq[nd] -= yq[c];
        }
    } else {
        double delta[CIPHER_MAXCP], ceq[CIPHER_MAXCP], un[CIPHER_MAXCP], bi[CIPHER_MAXCP];
        double mat[16], inv[16];
        for (int c = 0; c < ncp; c++) {
            ceq[c] = tseries(T, m.quad_ceq[c]);
            un[c] = tseries(T, m.unary[c]);
            bi[c] = tseries(T, m.quad_binary[c]);
        }
        for (int k = 0; k < 16; k++) { mat[k] = 0.0; inv[k] = 0.0; }
        for (int j = 0; j < nd; j++) {
            delta[j] = 0.5 * pot[j] + bi[nd] - 0.5 * (un[j] - un[nd]) + (bi[j] * ceq[j] - bi[nd] * ceq[nd]);
            mat[j * nd + j] += bi[j];
            for (int i = 0; i < nd; i++) mat[j * nd + i] += bi[nd];
        }
        invert_small(inv, mat, nd);
        matvec(y, inv, delta, nd);
        y[nd] = 1.0;
        for (int c = 0; c < nd; c++) y[nd] -= y[c];
    }
}

static __device__ __noinline__ void sitefrac_raw(const cipher_material &m, const double *pot, double T, int ncp, double *y)
{
    sitefrac_body<0, -1>(m, pot, T, ncp, y);
}

template <int NC, int MODEL, typename Mat>
static __device__ __forceinline__ void tangent_body(const Mat &m, const double *y, const double *pot, double T, int ncp_rt,
                                         double *tpot, double *tex, double *tT)
{
    const int ncp = NC > 0 ? NC : ncp_rt;
    const int model = MODEL >= 0 ? MODEL : m.model;

    const int nd = ncp - 1, nd2 = nd * nd;
    if (model == CIPHER_CHEM_NONE) {
        for (int c = 0; c < nd2; c++) { tpot[c] = 0.0; tex[c] = 0.0; }
        for (int c = 0; c < nd; c++) tT[c] = 0.0;
    } else if (model == CIPHER_CHEM_CALPHADDIS) {
        double RT = CIPHER_R_GAS * T, t[16];
        for (int k = 0; k < 16; k++) t[k] = 0.0;
        for (int j = 0; j < nd; j++) {
            t[j * nd + j] += y[j] / RT;
            for (int i = 0; i < nd; i++) t[j * nd + i] -= y[j] * y[i] / RT;
        }
        for (int c = 0; c < nd2; c++) { tpot[c] = t[c]; tex[c] = -t[c]; }
        for (int j = 0; j < nd; j++) tT[j] = 0.0;
        for (int j = 0; j < nd; j++) {
            for (int i = 0; i < nd; i++) tT[j] -= t[j * nd + i] * pot[i] / T;
        }
    } else if (model == CIPHER_CHEM_CALPHAD2SL) {
        double RT = CIPHER_R_GAS * T, tp[16], tq[16];
        const double *yp = y, *yq = y + ncp, *pp = pot, *pq = pot + nd;
        for (int k = 0; k < 16; k++) { tp[k] = 0.0; tq[k] = 0.0; }
        for (int j = 0; j < nd; j++) {
            tp[j * nd + j] += yp[j] / m.p / RT;
            tq[j * nd + j] += yq[j] / m.q / RT;
            for (int i = 0; i < nd; i++) {
                tp[j * nd + i] -= yp[j] * yp[i] / m.p / RT;
                tq[j * nd + i] -= yq[j] * yq[i] / m.q / RT;
            }
        }
        for (int c = 0; c < nd2; c++) {
            tpot[c] = tp[c]; tpot[nd2 + c] = tq[c];
            tex[c] = -tp[c]; tex[nd2 + c] = -tq[c];
        }
        for (int j = 0; j < 2 * nd; j++) tT[j] = 0.0;
        for (int j = 0; j < nd; j++) {
            for (int i = 0; i < nd; i++) {
                tT[j] -= tp[j * nd + i] * pp[i] / T;
                tT[nd + j] -= tq[j * nd + i] * pq[i] / T;
            }
        }
    } else {
        double delta[CIPHER_MAXCP], ceqT[CIPHER_MAXCP], unT[CIPHER_MAXCP], biT[CIPHER_MAXCP];
        double ceq[CIPHER_MAXCP], bi[CIPHER_MAXCP], mat[16], inv[16];
        for (int c = 0; c < ncp; c++) {
            ceqT[c] = tseries_dT(T, m.quad_ceq[c]);
            unT[c] = tseries_dT(T, m.unary[c]);
            biT[c] = tseries_dT(T, m.quad_binary[c]);
            ceq[c] = tseries(T, m.quad_ceq[c]);
            bi[c] = tseries(T, m.quad_binary[c]);
        }
        for (int k = 0; k < 16; k++) { mat[k] = 0.0; inv[k] = 0.0; }
        for (int j = 0; j < nd; j++) {
            mat[j * nd + j] += bi[j];
            for (int i = 0; i < nd; i++) mat[j * nd + i] += bi[nd];
        }
        invert_small(inv, mat, nd);
        for (int c = 0; c < nd2; c++) tpot[c] = inv[c] * 0.5;
        for (int c = 0; c < nd2; c++) tex[c] = 0.0;
        for (int j = 0; j < nd; j++)
            delta[j] = biT[nd] - 0.5 * (unT[j] - unT[nd])
                     + (biT[j] * ceq[j] + bi[j] * ceqT[j] - biT[nd] * ceq[nd] - bi[nd] * ceqT[nd]);
        matvec(tT, inv, delta, nd);
    }
}

static __device__ __noinline__ void tangent_raw(const cipher_material &m, const double *y, const double *pot, double T, int ncp,
                                   double *tpot, double *tex, double *tT)
{
    tangent_body<0, -1>(m, y, pot, T, ncp, tpot, tex, tT);
}

template <int NC, int MODEL, typename Mat>
static __device__ __forceinline__ void mobility_body(const Mat &m, const double *y, double T, int ncp_rt, double *M)
{
    const int ncp = NC > 0 ? NC : ncp_rt;
    const int model = MODEL >= 0 ? MODEL : m.model;

    if (model == CIPHER_CHEM_NONE) {
        for (int c = 0; c < ncp; c++) M[c] = 0.0;
    } else {
    for (int k = 0; k < ncp; k++) {
        const auto &mob = m.mobilityc[k];
        const auto *bin = mob.binary;
        double mig = 0.0;
        for (int j = 0; j < ncp; j++) {
            mig += y[j] * tseries(T, mob.unary[j]);
            for (int i = j + 1; i < ncp; i++, bin++)
                for (int r = 0; r < bin->n; r++)
                    mig += y[j] * y[i] * tseries(T, bin->h[r]) * ipow(y[j] - y[i], (unsigned)r);
        }
        M[k] = y[k] * mob.m0 / CIPHER_R_GAS / T * exp(mig / CIPHER_R_GAS / T);
    }
    }
}

static __device__ __noinline__ void mobility_raw(const cipher_material &m, const double *y, double T, int ncp, double *M)
{
    mobility_body<0, -1>(m, y, T, ncp, M);
}

/* the same over the evaluated tables (calphaddis, calphad2sl) */
static __device__ __noinline__ double energy_raw_v(const MatV &m, const double *y, double T, int ncp)
{
    return energy_body<0, -1>(m, y, T, ncp);
}

static __device__ __noinline__ void explicit_raw_v(const MatV &m, const double *y, double T, int ncp, double *mu)
{
    explicit_body<0, -1>(m, y, T, ncp, mu);
}

static __device__ __noinline__ void mobility_raw_v(const MatV &m, const double *y, double T, int ncp, double *M)
{
    mobility_body<0, -1>(m, y, T, ncp, M);
}

/* the evaluated tables of the material of `phase`, or NULL where the
 * phase's cell is at another temperature or its model is not CALPHAD */
__device__ __forceinline__ const MatV *matv_of(const ChemTables &t, int phase, int model)
{
    return (t.matv && (model == CIPHER_CHEM_CALPHADDIS || model == CIPHER_CHEM_CALPHAD2SL)) ? &t.matv[t.pmm[phase]]
                                                                                           : nullptr;
}

/* ---------------- per-phase wrappers with the molar-volume scaling ---------------- */
/* (src/material.c:480-490, 640-650, 701-727, 812-822, 995-1018, 1115-1120) */

__device__ inline double chemenergy(const ChemTables &t, int phase, const double *y, const double *mu, double T)
{
    const cipher_material &m = material_of(t, phase);
    const MatV *mv = matv_of(t, phase, m.model);
    double G = (mv ? energy_raw_v(*mv, y, T, t.ncp) : energy_raw(m, y, T, t.ncp)) / m.molarvolume;
    for (int s = 0; s < m.nsites; s++)
        for (int c = 0; c < t.ndp; c++) G -= mu[c] * m.stoichiometry[s] * y[s * t.ncp + c];
    return G;
}

__device__ inline void sitepot_explicit(const ChemTables &t, int phase, const double *y, double T, double *out)
{
    const cipher_material &m = material_of(t, phase);
    double full[2 * CIPHER_MAXCP];
    const MatV *mv = matv_of(t, phase, m.model);
    if (mv) explicit_raw_v(*mv, y, T, t.ncp, full);
    else explicit_raw(m, y, T, t.ncp, full);
    for (int s = 0; s < m.nsites; s++)
        for (int c = 0; c < t.ndp; c++)
            out[s * t.ndp + c] = (full[s * t.ncp + c] - full[s * t.ncp + t.ndp]) / m.molarvolume;
}

__device__ inline void sitepot_total(const ChemTables &t, int phase, const double *y, double T, double *out)
{
    const cipher_material &m = material_of(t, phase);
    double full[2 * CIPHER_MAXCP], im[2 * CIPHER_MAXCP], ex[2 * CIPHER_MAXCP];
    implicit_raw(m, y, T, t.ncp, full);
    for (int s = 0; s < m.nsites; s++)
        for (int c = 0; c < t.ndp; c++)
            im[s * t.ndp + c] = (full[s * t.ncp + c] - full[s * t.ncp + t.ndp]) / m.molarvolume;
    sitepot_explicit(t, phase, y, T, ex);
    for (int s = 0; s < m.nsites; s++)
        for (int c = 0; c < t.ndp; c++) out[s * t.ndp + c] = im[s * t.ndp + c] + ex[s * t.ndp + c];
}

__device__ inline void sitefrac(const ChemTables &t, int phase, const double *pot, double T, double *y)
{
    const cipher_material &m = material_of(t, phase);
    double scaled[2 * CIPHER_MAXCP];
    for (int s = 0; s < m.nsites; s++)
        for (int c = 0; c < t.ndp; c++) scaled[s * t.ndp + c] = m.molarvolume * pot[s * t.ndp + c];
    sitefrac_raw(m, scaled, T, t.ncp, y);
}

__device__ inline void sitefrac_tangent(const ChemTables &t, int phase, const double *y, const double *pot, double T,
                                        double *tpot, double *tex, double *tT)
{
    const cipher_material &m = material_of(t, phase);
    tangent_raw(m, y, pot, T, t.ncp, tpot, tex, tT);
    const int nd = t.ndp;
    for (int c = 0; c < m.nsites * nd * nd; c++) tpot[c] *= m.molarvolume;
    for (int c = 0; c < m.nsites * nd * nd; c++) tex[c] *= m.molarvolume;
    for (int c = 0; c < m.nsites * nd; c++) tT[c] *= m.molarvolume;
}

__device__ inline void mobility(const ChemTables &t, int phase, const double *y, double T, double *M)
{
    const cipher_material &m = material_of(t, phase);
    const MatV *mv = matv_of(t, phase, m.model);
    if (mv) mobility_raw_v(*mv, y, T, t.ncp, M);
    else mobility_raw(m, y, T, t.ncp, M);
    for (int c = 0; c < t.ncp; c++) M[c] *= m.molarvolume;
}

/* ---------------- the wrappers for one component count and model ---------------- */
/* The same operations as the wrappers above, with NC components and the
 * model's sublattice count model_nsites(MODEL) fixed at compile time and
 * the model bodies inlined: the single-phase kernels keep every array in
 * registers.  m is a material of that model. */

template <int NC, int MODEL, typename Mat>
__device__ __forceinline__ void sitefrac_m(const Mat &m, const double *pot, double T, double *y)
{
    constexpr int ND = NC - 1, NS = model_nsites(MODEL);
    double scaled[2 * CIPHER_MAXCP];
    for (int s = 0; s < NS; s++) {
        for (int c = 0; c < ND; c++) scaled[s * ND + c] = m.molarvolume * pot[s * ND + c];
    }
    sitefrac_body<NC, MODEL>(m, scaled, T, NC, y);
}

template <int NC, int MODEL, typename Mat>
__device__ __forceinline__ double chemenergy_m(const Mat &m, const double *y, const double *mu, double T)
{
    constexpr int ND = NC - 1, NS = model_nsites(MODEL);
    double G = energy_body<NC, MODEL>(m, y, T, NC) / m.molarvolume;
    for (int s = 0; s < NS; s++) {
        for (int c = 0; c < ND; c++) G -= mu[c] * m.stoichiometry[s] * y[s * NC + c];
    }
    return G;
}

template <int NC, int MODEL, typename Mat>
__device__ __forceinline__ void sitepot_explicit_m(const Mat &m, const double *y, double T, double *out)
{
    constexpr int ND = NC - 1, NS = model_nsites(MODEL);
    double full[2 * CIPHER_MAXCP];
    explicit_body<NC, MODEL>(m, y, T, NC, full);
    for (int s = 0; s < NS; s++) {
        for (int c = 0; c < ND; c++) out[s * ND + c] = (full[s * NC + c] - full[s * NC + ND]) / m.molarvolume;
    }
}

template <int NC, int MODEL, typename Mat>
__device__ __forceinline__ void sitefrac_tangent_m(const Mat &m, const double *y, const double *pot,
                                                   double T, double *tpot, double *tex, double *tT)
{
    constexpr int ND = NC - 1, NS = model_nsites(MODEL);
    tangent_body<NC, MODEL>(m, y, pot, T, NC, tpot, tex, tT);
    for (int c = 0; c < NS * ND * ND; c++) tpot[c] *= m.molarvolume;
    for (int c = 0; c < NS * ND * ND; c++) tex[c] *= m.molarvolume;
    for (int c = 0; c < NS * ND; c++) tT[c] *= m.molarvolume;
}

template <int NC, int MODEL, typename Mat>
__device__ __forceinline__ void mobility_m(const Mat &m, const double *y, double T, double *M)
{
    mobility_body<NC, MODEL>(m, y, T, NC, M);
    for (int c = 0; c < NC; c++) M[c] *= m.molarvolume;
}

/* the model calls of one phase: with NC > 0 and MODEL >= 0 the wrappers
 * above for that count and model (every material of the problem has the
 * model), reading the evaluated tables where the cell's temperature has
 * them (the CALPHAD energy, explicit potentials and mobility: the only
 * bodies that read T-series); else the general wrappers */
template <int NC, int MODEL>
struct PhaseModel {
    static constexpr bool kFixed = NC > 0 && MODEL >= 0;
    static constexpr bool kCalphad = MODEL == CIPHER_CHEM_CALPHADDIS || MODEL == CIPHER_CHEM_CALPHAD2SL;
    static __device__ __forceinline__ int nsites(const cipher_material &m)
    {
        if constexpr (kFixed) return model_nsites(MODEL);
        else return m.nsites;
    }
    static __device__ __forceinline__ void sitefrac(const ChemTables &t, int phase, const double *pot, double T, double *y)
    {
        if constexpr (kFixed) sitefrac_m<NC, MODEL>(material_of(t, phase), pot, T, y);
        else cipher::sitefrac(t, phase, pot, T, y);
    }
    static __device__ __forceinline__ double chemenergy(const ChemTables &t, int phase, const double *y, const double *mu,
                                                        double T)
    {
        if constexpr (kFixed && kCalphad) {
            /* the evaluated tables inline; a cell at another temperature
             * calls the general wrapper (the same operations) */
            if (t.matv) return chemenergy_m<NC, MODEL>(t.matv[t.pmm[phase]], y, mu, T);
            return cipher::chemenergy(t, phase, y, mu, T);
        } else if constexpr (kFixed) {
            return chemenergy_m<NC, MODEL>(material_of(t, phase), y, mu, T);
        } else {
            return cipher::chemenergy(t, phase, y, mu, T);
        }
    }
    static __device__ __forceinline__ void sitepot_explicit(const ChemTables &t, int phase, const double *y, double T,
                                                            double *out)
    {
        if constexpr (kFixed && kCalphad) {
            if (t.matv) sitepot_explicit_m<NC, MODEL>(t.matv[t.pmm[phase]], y, T, out);
            else cipher::sitepot_explicit(t, phase, y, T, out);
        } else if constexpr (kFixed) {
            sitepot_explicit_m<NC, MODEL>(material_of(t, phase), y, T, out);
        } else {
            cipher::sitepot_explicit(t, phase, y, T, out);
        }
    }
    static __device__ __forceinline__ void sitefrac_tangent(const ChemTables &t, int phase, const double *y,
                                                            const double *pot, double T, double *tpot, double *tex,
                                                            double *tT)
    {
        if constexpr (kFixed) sitefrac_tangent_m<NC, MODEL>(material_of(t, phase), y, pot, T, tpot, tex, tT);
        else cipher::sitefrac_tangent(t, phase, y, pot, T, tpot, tex, tT);
    }
    static __device__ __forceinline__ void mobility(const ChemTables &t, int phase, const double *y, double T, double *M)
    {
        if constexpr (kFixed && kCalphad) {
            if (t.matv) mobility_m<NC, MODEL>(t.matv[t.pmm[phase]], y, T, M);
            else cipher::mobility(t, phase, y, T, M);
        } else if constexpr (kFixed) {
            mobility_m<NC, MODEL>(material_of(t, phase), y, T, M);
        } else {
            cipher::mobility(t, phase, y, T, M);
        }
    }
};

}  // namespace cipher
