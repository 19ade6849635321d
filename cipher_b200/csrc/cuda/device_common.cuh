/*
 * device_common.cuh - device-side tables and helpers shared by the RHS and
 * PostStep kernels.
 *
 * Arithmetic that decides bit-exact outputs (phase sets) or that the FP64
 * path reproduces bit for bit follows the reference's operation order; the
 * FP64 translation units are compiled with --fmad=false so no multiply-add is
 * contracted (the reference's x86-64 build has no FMA either).
 */
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "cipher_problem.h"

#define CIPHER_PI_D 3.14159265358979323846264338327950288419716939937510582
#define CIPHER_PMAX 16

namespace cipher {

/* one interface, flattened for the device (INTERFACE, src/typedef.h:235-240) */
struct DevInterface {
    double width;
    double energy_m0, mobility_m0;
    cipher_tseries energy_act, mobility_act;
    int has_potential, has_mobilityc;
    double potential[CIPHER_MAXCP];
    double mobilityc[CIPHER_MAXCP];
    int nsources;
    cipher_source sources[CIPHER_MAXSRC];
    /* anisotropy (IENERGY / IMOBILITY dir, val, n): unit directions [n][dim] */
    int energy_n, mobility_n;
    double energy_dir[CIPHER_MAXDIR * 3], energy_val[CIPHER_MAXDIR];
    double mobility_dir[CIPHER_MAXDIR * 3], mobility_val[CIPHER_MAXDIR];
};

/* A T-series evaluated at one temperature, and the CALPHAD model tables of
 * a material with every series evaluated (rhs_general.cu: k_evaluate): the
 * fields the calphaddis and calphad2sl model bodies read (models.cuh), laid
 * out densely - a cipher_rk spends 568 bytes on what an order count and one
 * value per order say here. */
struct TsV {
    double v;
};
struct RkV {
    int32_t n;
    int32_t i[CIPHER_MAXRK];
    TsV h[CIPHER_MAXRK];
};
struct MobV {
    double m0;
    TsV unary[CIPHER_MAXCP];
    RkV binary[CIPHER_MAXBIN];
};
struct MatV {
    int32_t model;
    double p, q, molarvolume, stoichiometry[2];
    TsV ref, unary[CIPHER_MAXCP * CIPHER_MAXCP];
    RkV binary[CIPHER_MAXRKTAB], ternary[CIPHER_MAXRKTAB], binaryq[CIPHER_MAXRKTAB], ternaryq[CIPHER_MAXRKTAB];
    MobV mobilityc[CIPHER_MAXCP];
    TsV quad_ceq[CIPHER_MAXCP], quad_binary[CIPHER_MAXCP];   /* for the quadratic branches; never read */
};

/* material tables on the device: the host structs of cipher_problem.h
 * copied unchanged, and the phase -> material map */
struct ChemTables {
    const cipher_material *mat;      /* [nmat] */
    const int32_t *pmm;              /* [npf] */
    int ncp, ndp, nmat;
    /* the CALPHAD materials with every T-series replaced by its value at
     * *tspec (rhs_general.cu: k_specialise), or NULL */
    const cipher_material *spec;
    const double *tspec;
    /* the same materials as MatV at *tspec (NULL: none) */
    const MatV *matv_tab;
    /* matv_tab in the tables chem_at returns for a cell at *tspec, else
     * NULL: the model wrappers read the evaluated tables through this */
    const MatV *matv;
};

/* the tables a cell at temperature T reads: the specialised copy when it
 * was made for exactly this T (same values, computed by the same tseries) */
__device__ __forceinline__ ChemTables chem_at(const ChemTables &t, double T)
{
    ChemTables r = t;
    r.matv = nullptr;
    if (t.spec && T == *t.tspec) {
        r.mat = t.spec;
        r.matv = t.matv_tab;
    }
    return r;
}

/* error flags raised by kernels (bit mask); never a trap */
enum : int {
    ERR_CAP = 1,        /* active-set superset above P */
    ERR_BADSET = 2,     /* n > P or an id >= npf in the input state */
    ERR_NONFINITE = 4,
};

/* exponentiation by squaring, as the reference's FastPow (src/utility.c:112-124) */
__device__ __forceinline__ double ipow(double b, unsigned e)
{
    double r = 1.0;
    while (e) {
        if (e & 1u) r *= b;
        e >>= 1;
        b *= b;
    }
    return r;
}

/* T-series sum (src/utility.c:48-62) */
__device__ inline double tseries(double T, const cipher_tseries &s)
{
    double r = 0.0;
    for (int i = 0; i < s.n; i++) {
        int e = s.exp[i];
        if (e > 0) r += s.coeff[i] * ipow(T, (unsigned)e);
        else if (e < 0) r += s.coeff[i] / ipow(T, (unsigned)(-e));
        else r += s.coeff[i];
    }
    if (fabs(s.logcoeff) > 0.0) r += s.logcoeff * T * log(T);
    return r;
}

/* an evaluated series: tseries(T, s) of the specialised series it was made
 * from, bit for bit */
__device__ __forceinline__ double tseries(double, const TsV &s) { return s.v; }

/* pair properties sigma, m, w of an interface at temperature T
 * (src/cipher.c:422-471 without anisotropy) */
__device__ inline void interface_props(const DevInterface &itf, double T, double &sig, double &mob, double &wid)
{
    sig = 1.0;
    mob = 1.0;
    sig *= itf.energy_m0;
    if (itf.energy_act.n) sig *= exp(tseries(T, itf.energy_act) / CIPHER_R_GAS / T);
    mob *= itf.mobility_m0;
    if (itf.mobility_act.n) mob *= exp(tseries(T, itf.mobility_act) / CIPHER_R_GAS / T);
    wid = itf.width;
}

/* the same with the anisotropy of the pair's interface normal u (unit, or
 * zero where the gradients cancel): sigma and m start from
 * 1 + sum_dir (u . dir)^4 val_dir before the prefactor and the activation
 * term (src/cipher.c:427-460) */
__device__ inline void interface_props_aniso(const DevInterface &itf, double T, const double *u, int dim, double &sig,
                                             double &mob, double &wid)
{
    sig = 1.0;
    mob = 1.0;
    for (int k = 0; k < itf.energy_n; k++) {
        double dot = 0.0;
        for (int d = 0; d < dim; d++) dot += u[d] * itf.energy_dir[dim * k + d];
        sig += ipow(dot, 4) * itf.energy_val[k];
    }
    for (int k = 0; k < itf.mobility_n; k++) {
        double dot = 0.0;
        for (int d = 0; d < dim; d++) dot += u[d] * itf.mobility_dir[dim * k + d];
        mob += ipow(dot, 4) * itf.mobility_val[k];
    }
    sig *= itf.energy_m0;
    if (itf.energy_act.n) sig *= exp(tseries(T, itf.energy_act) / CIPHER_R_GAS / T);
    mob *= itf.mobility_m0;
    if (itf.mobility_act.n) mob *= exp(tseries(T, itf.mobility_act) / CIPHER_R_GAS / T);
    wid = itf.width;
}

}  // namespace cipher
