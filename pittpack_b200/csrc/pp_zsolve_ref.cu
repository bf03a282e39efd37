// The reference's alternate z solvers, reproduced as its CPU build computes
// them (parity modes PP_ZSOLVE_REF_PCR and PP_ZSOLVE_REF_CRP): SOLUTIONMETHOD
// 1 and 2 of src/pencilDcmp.cpp:6102-6148.
//
//   PCR   solvePCR (src/pencilDcmp.cpp:5239-5270): the system divided by
//         lambda (fillInArrayContigNormalize :5320-5345,
//         imposeBoundaryonContainer :5372-5401, offDiagNormalize :5406-5452,
//         imposeBoundaryonOffDiag :5457-5481), then TriDiag::pcr
//         (src/triDiag.cpp:1442-1542).  That routine gathers each row's
//         neighbours into per-lane arrays of an OpenACC vector; compiled for
//         the CPU they are arrays indexed by row / VECLENGTH (256), so every
//         row of a 256-row block is updated with the neighbours of the
//         block's last row, and the solution comes out constant along z.
//         Reproduced for Dirichlet / Neumann ends and nz <= 256 not a power
//         of two, where that computation reads within bounds.
//   CR-P  solveCRP (src/pencilDcmp.cpp:5275-5315) -> TriDiag::crp
//         (src/triDiag.cpp:1285-1437): cyclic reduction of the
//         constant-coefficient system (diagonal 1, off-diagonals 1 / lambda;
//         the Dirichlet ghost-cell diagonal is not applied, the end rows are
//         divided by lambda) to a 3 x 3 system and back-substitution;
//         nz = 2^L - 1, Dirichlet ends.
//
// One thread per (system, real or imaginary part), on the [k][ky][kx]
// spectrum in place; the arithmetic is written with round-to-nearest
// intrinsics in the reference's operation order (no contraction into FMA).
#include "../../include/pittpack_b200.h"
#include "pp_common.cuh"
#include "pp_kernels.h"

namespace {

PP_D double dm(double a, double b) { return __dmul_rn(a, b); }
PP_D double da(double a, double b) { return __dadd_rn(a, b); }
PP_D double ds(double a, double b) { return __dsub_rn(a, b); }
PP_D double dd(double a, double b) { return __ddiv_rn(a, b); }

// element k of the column of thread (system, part)
struct RefCol {
    double* p;
    long stride;
    PP_D double& operator[](int k) const { return p[k * stride]; }
};

// the pcr recurrence of one system (n <= 256: one block of 256 rows)
PP_D void ref_pcr(int n, double* a, double* c, const RefCol& d)
{
    int level = 0;
    while ((2 << level) <= n) ++level;  // floor(log2 n)
    level += 1;
    for (int p = 0; p < level; p++) {
        const int s = 1 << p;
        // the neighbours of the block's last row (i = n - 1: i - s >= 0 and
        // i + s >= n for every s < n)
        const int i = n - 1;
        const double a0 = a[i], a1 = a[i - s], c0 = c[i], c1 = c[i - s];
        const double d0 = d[i], d1 = d[i - s];
        const double r = dd(1., ds(ds(1., dm(a0, c1)), dm(c0, 0.0)));
        const double an = dm(dm(-r, a0), a1);
        const double cn = dm(dm(-r, c0), 0.0);
        const double dn = dm(r, ds(ds(d0, dm(a0, d1)), dm(c0, 0.0)));
        for (int k = 0; k < n; k++) {
            a[k] = an;
            c[k] = cn;
            d[k] = dn;
        }
    }
}

// the three-row Thomas of crp (thomasLowMem, src/triDiag.cpp:1891-1950, b = 1)
PP_D void ref_thomas3(double a1, double a2, double c0, double c1, double* r)
{
    double bet = 1.0;
    r[0] = dd(r[0], bet);
    const double g1 = dd(c0, bet);
    bet = ds(1.0, dm(a1, g1));
    r[1] = dd(ds(r[1], dm(a1, r[0])), bet);
    const double g2 = dd(c1, bet);
    bet = ds(1.0, dm(a2, g2));
    r[2] = dd(ds(r[2], dm(a2, r[1])), bet);
    r[1] = ds(r[1], dm(g2, r[2]));
    r[0] = ds(r[0], dm(g1, r[1]));
}

PP_D void ref_crp(int n, double offdiag, const RefCol& rhs)
{
    int level = 0;
    while ((2 << level) <= n) ++level;  // floor(log2 n)
    double tmpA[16], tmpC[16];
    int m = n;
    tmpA[0] = offdiag;
    tmpC[0] = offdiag;
    for (int i = 0; i < level - 1; i++) {
        const int d1 = 1 << (i + 1);
        m = m >> 1;
        const double a0 = tmpA[i], c0 = tmpC[i];
        const double cte = ds(1., dm(dm(2., a0), c0));
        for (int j = 0; j < m; j++) {
            const int ind0 = d1 * j + (d1 - 1);
            const int im1 = ind0 - d1 / 2, ip1 = ind0 + d1 / 2;
            rhs[ind0] = dd(da(da(dm(rhs[im1], -a0), rhs[ind0]), dm(rhs[ip1], -c0)), cte);
        }
        tmpA[i + 1] = dd(dm(-a0, a0), cte);
        tmpC[i + 1] = dd(dm(-c0, c0), cte);
    }
    {
        const int d1 = 1 << level;
        const int ind0 = d1 - 1, im1 = ind0 - d1 / 2, ip1 = ind0 + d1 / 2;
        double t[3] = {rhs[im1], rhs[ind0], rhs[ip1]};
        ref_thomas3(tmpA[level - 1], tmpA[level - 1], tmpC[level - 1], tmpC[level - 1], t);
        rhs[ind0] = t[1];
        rhs[im1] = t[0];
        rhs[ip1] = t[2];
    }
    m = 3;
    for (int i = level - 1; i > 0; i--) {
        const int d0 = 1 << i;
        for (int j = 0; j < m; j++) {
            const int q = d0 * j + (d0 - 1) - d0 / 2;
            rhs[q] = ds(rhs[q], dm(tmpA[i - 1], rhs[d0 * j + (d0 - 1)]));
        }
        for (int j = 0; j < m; j++) {
            const int q = d0 * j + (d0 - 1) + d0 / 2;
            rhs[q] = ds(rhs[q], dm(tmpC[i - 1], rhs[d0 * j + (d0 - 1)]));
        }
        m = (1 << (level - i + 2)) - 1;
    }
}

__global__ void zsolve_ref_kernel(PPZRefArgs a)
{
    const long systems = (long)a.nx * a.ny;
    const long items = systems * a.parts;
    for (long it = blockIdx.x * (long)blockDim.x + threadIdx.x; it < items; it += (long)gridDim.x * blockDim.x) {
        const long sys = it / a.parts;
        const int part = (int)(it - sys * a.parts);
        const int ky = (int)(sys / a.nx);
        const int kx = (int)(sys - (long)ky * a.nx);
        const int nz = a.nz;
        // getEigenVal (src/pencilDcmp.cpp:4393-4417) from the per-direction parts
        const double eig = da(da(-2.0, dm(a.ax[kx], a.Cx)), dm(a.ay[ky], a.Cy));
        const long plane = (long)a.nx * a.ny;
        RefCol r{a.data + (long)a.parts * sys + part, (long)a.parts * plane};
        const double eigInv = dd(1., eig);
        const double r0 = r[0], rn = r[nz - 1];
        for (int k = 1; k < nz - 1; k++) r[k] = dm(r[k], eigInv);
        if (a.method == PP_ZSOLVE_REF_CRP) {
            r[0] = dd(r0, eig);
            r[nz - 1] = dd(rn, eig);
            ref_crp(nz, dd(1., eig), r);
            continue;
        }
        const double em1 = ds(eig, 1.), ep1 = da(eig, 1.);
        r[0] = dd(r0, a.zlo == PP_Z_DIRICHLET ? em1 : ep1);
        r[nz - 1] = dd(rn, a.zhi == PP_Z_DIRICHLET ? em1 : ep1);
        double lower[256], upper[256];
        for (int k = 1; k < nz; k++) lower[k] = eigInv;
        for (int k = 0; k < nz - 1; k++) upper[k] = eigInv;
        lower[0] = 0.0;
        upper[nz - 1] = 0.0;
        upper[0] = dd(1., a.zlo == PP_Z_DIRICHLET ? em1 : ep1);
        lower[nz - 1] = dd(1., a.zhi == PP_Z_DIRICHLET ? em1 : ep1);
        ref_pcr(nz, lower, upper, r);
    }
}

}  // namespace

bool pp_zsolve_ref_defined(int method, int nz, int zlo, int zhi)
{
    if (method == PP_ZSOLVE_REF_PCR)
        return zlo != PP_Z_PERIODIC && zhi != PP_Z_PERIODIC && nz >= 3 && nz <= 256 && (nz & (nz - 1)) != 0;
    if (method == PP_ZSOLVE_REF_CRP)
        return zlo == PP_Z_DIRICHLET && zhi == PP_Z_DIRICHLET && nz >= 3 && nz <= 32767 && ((nz + 1) & nz) == 0;
    return false;
}

cudaError_t pp_launch_zsolve_ref(const PPZRefArgs& a, cudaStream_t st)
{
    if (!pp_zsolve_ref_defined(a.method, a.nz, a.zlo, a.zhi)) return cudaErrorInvalidValue;
    const long items = (long)a.nx * a.ny * a.parts;
    const long blocks = (items + 127) / 128;
    zsolve_ref_kernel<<<(unsigned)(blocks < 148L * 32 ? blocks : 148L * 32), 128, 0, st>>>(a);
    return cudaGetLastError();
}
