// Table values shared by the handle path (computed on the host at set-up)
// and the allocation-free solve (computed on the device into its fixed
// array): one definition of each formula, compiled for both sides.
#pragma once

#include <math.h>

#include "pp_common.cuh"

// the reference's constant (src/include/params.h: const double pi)
#define PP_REF_PI 3.1415926535897932384

// Family twiddle k of a DCT/DST direction of length n: the reference's angle
// theta = (pi / 2 / N) k with its pi constant (postprocessSignalDCT10,
// src/signalProc.cpp:32-71); (cos theta, sin theta)
PP_HD double2 pp_family_twiddle(int n, int k)
{
    const double theta = (PP_REF_PI / 2. / n) * k;
    return make_double2(cos(theta), sin(theta));
}

// Eigenvalue part of one direction (setEigenVal src/pencilDcmp.cpp:3533-3576,
// getEigenVal 4393-4417): -2 + 2 cos((k + num) f / (n + den)) with num = 1 for
// D-D, 1/2 for the quarter-wave N-D / D-N families, f = 2 pi for P-P, else pi
PP_HD double pp_eigen_part(int n, int kind, int k)
{
    double num = 0.0, den = 0.0, freq = PP_REF_PI;
    if (kind == PP_KIND_DST2) num = 1.0;
    else if (kind == PP_KIND_FFT) freq = 2. * PP_REF_PI;
    else if (pp_kind_is_quarter(kind)) num = 0.5;
    return -2.0 + 2. * cos((k + num) * freq / (n + den));
}

// The manufactured-solution Dirichlet faces that modifyRhsDirichlet
// (src/pencilDcmp.cpp:4623-4835) subtracts from the dz^2-scaled RHS, with
// exactValue (src/pencilDcmp.cpp:1837-1866) and the tags of extractTag
// (src/pencilDcmp.cpp:3636-3668).  Face slots: 0 z-min, 1 z-max ([j][i]),
// 2 x-min, 3 x-max ([k][j]), 4 y-min, 5 y-max ([k][i]).
struct PPMmsFaces {
    int nx, ny, nz;
    double Xa, Ya, Za;
    double c1, c2, c3;   // cell sizes
    double omega[3];     // 1 pi, 2 pi, 3 pi
    int t0, t1, t2;      // tags of x, y, z
};

PP_HD double pp_exact_value(double omega, double x, int tg)
{
    if (fabs(omega) < 1.0e-6) return 1.0;
    if (tg == 0 || tg == -1 || tg == -2) return sin(omega * x);
    if (tg == 1) return cos(omega * x);
    return 0.0;
}

// coordinates the reference evaluates on each face (cell centres, shift 1,
// and the face plane itself)
PP_HD double pp_mms_x(const PPMmsFaces& p, int i) { return p.Xa + i * p.c1 + 1.0 * p.c1 * .5; }
PP_HD double pp_mms_y(const PPMmsFaces& p, int j) { return p.Ya + j * p.c2 + 1.0 * p.c2 * 0.5; }
PP_HD double pp_mms_z(const PPMmsFaces& p, int k) { return p.Za + k * p.c3 + 1.0 * p.c3 * .5; }
PP_HD double pp_mms_face_plane(const PPMmsFaces& p, int slot)
{
    switch (slot) {
    case 0: return p.Za;
    case 1: return p.Za + (p.nz - 1) * p.c3 + p.c3;
    case 2: return p.Xa;
    case 3: return p.Xa + ((p.nx - 1) + 1) * p.c1;
    case 4: return p.Ya;
    default: return p.Ya + ((p.ny - 1) + 1) * p.c2;
    }
}

// value of face `slot` at its position (a, b): (i, j) on z faces, (j, k) on
// x faces, (i, k) on y faces
PP_HD double pp_mms_face_value(const PPMmsFaces& p, int slot, int a, int b)
{
    const double w = pp_mms_face_plane(p, slot);
    if (slot < 2)
        return 2. * pp_exact_value(p.omega[0], pp_mms_x(p, a), p.t0) * pp_exact_value(p.omega[1], pp_mms_y(p, b), p.t1) *
               pp_exact_value(p.omega[2], w, p.t2);
    if (slot < 4)
        return 2. * pp_exact_value(p.omega[0], w, p.t0) * pp_exact_value(p.omega[1], pp_mms_y(p, a), p.t1) *
               pp_exact_value(p.omega[2], pp_mms_z(p, b), p.t2);
    return 2. * pp_exact_value(p.omega[0], pp_mms_x(p, a), p.t0) * pp_exact_value(p.omega[1], w, p.t1) *
           pp_exact_value(p.omega[2], pp_mms_z(p, b), p.t2);
}

// extent (a, b) of a face slot
PP_HD void pp_mms_face_dims(const PPMmsFaces& p, int slot, int* na, int* nb)
{
    if (slot < 2) {
        *na = p.nx;
        *nb = p.ny;
    } else if (slot < 4) {
        *na = p.ny;
        *nb = p.nz;
    } else {
        *na = p.nx;
        *nb = p.nz;
    }
}

// FFT length of a direction.  The quarter-wave families (DCT-IV / DST-IV) of
// even length n run one n/2-point complex FFT of the paired, pre-twiddled
// line; of odd length n, one 2n-point FFT of the pre-twiddled line padded
// with n zeros:
//   X_k = c Re[ e^{-i pi (2k+1)/(4n)} sum_{m<n} (x_m e^{-i pi m/(2n)}) e^{-2 pi i m k/(2n)} ].
// Every other family: n.
PP_HD int pp_fft_len(int n, int kind)
{
    if (!pp_kind_is_quarter(kind)) return n;
    return (n & 1) ? 2 * n : n / 2;
}

// entries of a direction's family-twiddle table: the DCT/DST families' n
// (theta_k); the quarter-wave families' pre- and post-twiddles, n / 2 each
// (even n) or n each (odd n)
PP_HD int pp_family_table_len(int n, int kind) { return (pp_kind_is_quarter(kind) && (n & 1)) ? 2 * n : n; }

// the quarter-wave families' twiddle table entry idx, as the fraction f of pi
// in e^{-i pi f}: even n, idx < n/2: m / n (pre, m = idx), else
// (4p + 1) / (4n) (post, p = idx - n/2); odd n, idx < n: m / (2n), else
// (2k + 1) / (4n) (k = idx - n)
PP_HD void pp_quarter_angle(int n, int idx, long* num, long* den)
{
    if (n & 1) {
        if (idx < n) {
            *num = idx;
            *den = 2L * n;
        } else {
            *num = 2L * (idx - n) + 1;
            *den = 4L * n;
        }
    } else {
        const int h = n / 2;
        if (idx < h) {
            *num = idx;
            *den = n;
        } else {
            *num = 4L * (idx - h) + 1;
            *den = 4L * n;
        }
    }
}
