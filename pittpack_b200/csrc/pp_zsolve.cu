// Batched z-direction tridiagonal solve.
//
// The reference gathers each strided z-line into a buffer and runs a serial
// Thomas sweep per line (solveThmBatch, src/pencilDcmp.cpp:5066-5105 ->
// TriDiag::thomasLowMem, src/triDiag.cpp:1693-1822; periodic z through
// TriDiag::shermanMorrisonThomas, src/triDiag.cpp:1961-2108).  The system of
// mode (kx, ky) is
//     x_{k-1} + lambda x_k + x_{k+1} = r_k,   lambda = getEigenVal(ky, kx)
//     (src/pencilDcmp.cpp:4393-4417), computed here on the fly per system,
// with the ends modified by the z boundary: Dirichlet b = lambda - 1, Neumann
// b = lambda + 1 (src/triDiag.cpp:1733-1751), periodic: cyclic corners 1.
// Zero mode (|lambda + 2| < 1e-10): the reference replaces row 0 by x_0 = r_0
// (src/triDiag.cpp:1753-1776); for periodic z it solves the cyclic system
// with row 0 replaced by x_0 + x_{N-1} = (r_0 + r_{N-1}) / 2
// (shermanMorrisonThomasV1, src/triDiag.cpp:2112-2255).
//
// B200 layout and algorithm:
//   * a CTA owns TS adjacent kx columns of one ky row; it reads the TS x nz
//     tile into shared memory, solves, and writes the tile back: in the
//     z-tiled layout (the tile one contiguous block) with one bulk copy per
//     lane's block of rows where the rows live in registers, else with
//     coalesced row segments (rows skewed by one slot every 16 to spread
//     banks);
//   * a group of P lanes (P = 32 / systems per warp) solves one system by the
//     partition method: lane L owns a contiguous block of M ~ nz/P rows and
//     eliminates it so that every interior unknown is expressed through the
//     block's first and last unknown (a forward sweep, a backward sweep for
//     the first row, a recovery sweep), leaving two equations per lane; the
//     rows stay in registers where the counts allow.  Interior rows have the
//     same coefficients in every block, so the pivots and spikes of a block
//     depend only on lambda; the CTA builds them into a shared table (one
//     reciprocal per entry) that every lane reads, and the sweeps divide only
//     on the system's last row;
//   * eliminating each lane's first unknown leaves a P-row tridiagonal system
//     in the lanes' last unknowns, solved by parallel cyclic reduction over
//     warp shuffles (periodic systems through Sherman-Morrison); each lane
//     then recovers its interior rows;
//   * where every lane keeps exactly 10, 12, 16, 20, 24 or 32 rows in registers, they form two
//     blocks of half that length whose sweeps run side by side (two
//     independent FP64 recurrences per lane: the sweeps are bound by the
//     latency of their dependent operations), and one more elimination step
//     on the lane reduces the two blocks' rows to one before the shuffles.
#include <type_traits>

#include "pp_common.cuh"
#include "pp_kernels.h"

namespace {

PP_D double zmul(double s, double x) { return s * x; }
PP_D double2 zmul(double s, double2 x) { return make_double2(s * x.x, s * x.y); }
PP_D double zsub(double a, double b) { return a - b; }
PP_D double2 zsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
PP_D double zadd(double a, double b) { return a + b; }
PP_D double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
template <typename T>
PP_D T zzero();
template <>
PP_D double zzero<double>() { return 0.0; }
template <>
PP_D double2 zzero<double2>() { return make_double2(0.0, 0.0); }

// warp shuffles within segments of w lanes (one lane group)
PP_D double zshfl(double v, int src, int w) { return __shfl_sync(0xffffffffu, v, src, w); }
PP_D double2 zshfl(double2 v, int src, int w)
{
    return make_double2(__shfl_sync(0xffffffffu, v.x, src, w), __shfl_sync(0xffffffffu, v.y, src, w));
}
PP_D double zshfl_up(double v, int d, int w) { return __shfl_up_sync(0xffffffffu, v, d, w); }
PP_D double2 zshfl_up(double2 v, int d, int w)
{
    return make_double2(__shfl_up_sync(0xffffffffu, v.x, d, w), __shfl_up_sync(0xffffffffu, v.y, d, w));
}
PP_D double zshfl_down(double v, int d, int w) { return __shfl_down_sync(0xffffffffu, v, d, w); }
PP_D double2 zshfl_down(double2 v, int d, int w)
{
    return make_double2(__shfl_down_sync(0xffffffffu, v.x, d, w), __shfl_down_sync(0xffffffffu, v.y, d, w));
}

// asynchronous global -> shared copies (LDGSTS): no register staging, every
// copy of a tile in flight at once
PP_D void cp_async8(void* smem, const void* gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
PP_D void cp_async16(void* smem, const void* gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
PP_D void cp_async4(void* smem, const void* gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
PP_D void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// skewed position of row k inside a system's column of the tile
PP_HD int zpos(int k) { return k + (k >> 4); }
PP_HD int zpitch(int nz) { return (zpos(nz - 1) + 1) | 1; }

// Thread order of the tile's load and store (element e of the TS x nz tile ->
// system s, row k).  Shared memory serves a warp's 8-byte accesses in two
// phases of 16 threads (16-byte ones in four of 8), so a phase of W threads
// takes the W / TS rows k0 + r TS (r < W / TS) of its TS systems: with an odd
// column pitch p the slots s p + k0 + r TS are W distinct banks.  The rows of
// a phase pair then lie in two 128-byte segments of global memory.
PP_D void zt_elem(int e, int TS, int lts, int esz, int* s, int* k)
{
    const int lw = esz == 16 ? 3 : 4;
    const int W = 1 << lw;
    if (TS > W) {
        *k = e >> lts;
        *s = e & (TS - 1);
        return;
    }
    const int blk = e >> (lw + lts);        // W rows of the tile
    const int f = e & ((W << lts) - 1);
    const int ph = f >> lw;                 // phase: rows ph + r TS
    const int jj = f & (W - 1);
    *s = jj & (TS - 1);
    *k = (blk << lw) + ph + ((jj >> lts) << lts);
}
// f(s, k) for every element of the tile (s < ts, k < nz) in that order.  A
// thread keeps its system and steps its row: by blockDim.x / TS when the CTA
// covers whole periods of the order (W TS elements, TS where TS > W); else
// by blockDim.x / W within a period (R = period / blockDim.x steps) and on
// to the next period's W rows.  blockDim.x is a power of two >= 32.
template <typename T, typename F>
PP_D void zt_each(int TS, int lts, int nz, int ts, F f)
{
    const int esz = (int)sizeof(T);
    const int W = esz == 16 ? 8 : 16;
    const int period = TS > W ? TS : W * TS;
    int s, k;
    zt_elem(threadIdx.x, TS, lts, esz, &s, &k);
    if (s >= ts) return;
    if ((int)blockDim.x >= period) {
        const int kst = blockDim.x >> lts;
        for (; k < nz; k += kst) f(s, k);
    } else {
        const int R = period / blockDim.x, dk = blockDim.x / W;
        for (int r = 0; k < nz;) {
            f(s, k);
            if (++r == R) {
                r = 0;
                k += W - (R - 1) * dk;
            } else {
                k += dk;
            }
        }
    }
}

// The reduced system of a lane group, one row per lane L in the lanes' last
// unknowns l:  ra l_{L-1} + rb l_L + rc l_{L+1} = rd,  lane indices wrapping
// (periodic z; otherwise ra = 0 on the first lane and rc = 0 on the last).
// Solved by parallel cyclic reduction over warp shuffles, the periodic one
// through Sherman-Morrison; returns l_L.
template <typename T>
PP_D T zsolve_reduced(double ra, double rb, double rc, T rd, int lane, int P, bool periodic)
{
    if (P == 1)  // one row: its neighbours on both sides are itself
        return zmul(1.0 / (ra + rb + rc), rd);
    {
        const double inv = 1.0 / rb;
        ra *= inv;
        rc *= inv;
        rd = zmul(inv, rd);
    }
    double ru = 0.0, beta = 0.0;
    const double gam = -1.0;
    if (periodic) {
        // the corners move into u v^T with u = (gam, 0, .., alpha),
        // v = (1, 0, .., beta / gam): beta = a_0, alpha = c_{P-1}
        beta = zshfl(ra, 0, P);
        const double alpha = zshfl(rc, P - 1, P);
        if (lane == 0) {
            const double b0 = 1.0 - gam;
            ra = 0.0;
            rc /= b0;
            rd = zmul(1.0 / b0, rd);
            ru = gam / b0;
        }
        if (lane == P - 1) {
            const double bl = 1.0 - alpha * beta / gam;
            rc = 0.0;
            ra /= bl;
            rd = zmul(1.0 / bl, rd);
            ru = alpha / bl;
        }
    }
    for (int st = 1; st < P; st <<= 1) {
        const bool hp = lane >= st, hn = lane + st < P;
        double ap = zshfl_up(ra, st, P), cp = zshfl_up(rc, st, P);
        T dp = zshfl_up(rd, st, P);
        double an = zshfl_down(ra, st, P), cn = zshfl_down(rc, st, P);
        T dnx = zshfl_down(rd, st, P);
        if (!hp) {
            ap = cp = 0.0;
            dp = zzero<T>();
        }
        if (!hn) {
            an = cn = 0.0;
            dnx = zzero<T>();
        }
        const double inv = 1.0 / (1.0 - ra * cp - rc * an);
        if (periodic) {
            const double up = zshfl_up(ru, st, P), un = zshfl_down(ru, st, P);
            ru = (ru - ra * (hp ? up : 0.0) - rc * (hn ? un : 0.0)) * inv;
        }
        rd = zmul(inv, zsub(zsub(rd, zmul(ra, dp)), zmul(rc, dnx)));
        ra = -ra * ap * inv;
        rc = -rc * cn * inv;
    }
    if (!periodic) return rd;
    // fact = (y_0 + (beta/gam) y_{P-1}) / (1 + z_0 + (beta/gam) z_{P-1})
    const double bg = beta / gam;
    const T y0 = zshfl(rd, 0, P), yl = zshfl(rd, P - 1, P);
    const double z0 = zshfl(ru, 0, P), zl = zshfl(ru, P - 1, P);
    const T fact = zmul(1.0 / (1.0 + z0 + bg * zl), zadd(y0, zmul(bg, yl)));
    return zsub(rd, zmul(ru, fact));
}

// The partition solve of one system by its lane group with each lane's MT
// rows (registers xr, MT = nz / P) split into two blocks of H = MT / 2 rows,
// A = xr[0, H) and B = xr[H, MT), whose sweeps run side by side (two
// independent recurrences per lane instead of one of twice the length).
// Every block is eliminated as in the one-block solve: forward sweep, spike
// row of the block's first unknown f, its last row E1 -- leaving
//   E0: f + e0a l_prev + e0c l = e0d,   E1: e1a f + l + e1c f_next = e1d
// per block, l the block's last unknown and prev / next the adjacent blocks
// (B of the previous lane, B of this lane for A; A of this lane, A of the
// next lane for B).  Eliminating every f leaves one row per block in the l's;
// eliminating l_A (its neighbours l_B of the previous lane and of this one)
// leaves one row per lane in the l_B's, solved by zsolve_reduced; l_A, both
// f's and the blocks' interior rows follow.  tab holds the interior pivots of
// a block of H rows (gamma_i, alpha_i, i < H); d0 is row 0's right-hand side
// (after the periodic zero-mode averaging); row 0 of the system is the first
// row of A on lane 0 and row nz - 1 the last row of B on lane P - 1.
template <int MT, typename T>
PP_D void zsolve_split(T (&xr)[MT], const double2* tab, T d0, bool live, bool clear, int lane, int P,
                       bool periodic, double lam, double A0, double B0, double C0, double AN, double BN,
                       double CN)
{
    constexpr int H = MT / 2;
    static_assert(H >= 4, "blocks of at least four rows");
    const double* tg = reinterpret_cast<const double*>(tab);  // gamma_i = tg[2i], alpha_i = tg[2i+1]
    const bool last = lane == P - 1;
    // ---- forward sweeps of A and B ----------------------------------------------------
    T dA = zzero<T>(), dB = zzero<T>();
    double gA = 0.0, gB = 0.0, aA = 0.0, aB = 0.0;
    if (live) {
        bool lastB = false;
#pragma unroll
        for (int i = 1; i < H; ++i) {
            const double ga = tg[2 * i];
            const T nA = (i == 1) ? zmul(ga, xr[i]) : zmul(ga, zsub(xr[i], dA));
            T nB;
            if (i == H - 1 && last) {
                // the system's last row closes B on the last lane
                const double p = 1.0 / (BN - AN * gB);
                aB = -AN * tg[2 * (i - 1) + 1] * p;
                gB = CN * p;
                nB = zmul(p, zsub(xr[H + i], zmul(AN, dB)));
                lastB = true;
            } else {
                nB = (i == 1) ? zmul(ga, xr[H + i]) : zmul(ga, zsub(xr[H + i], dB));
                gB = ga;
            }
            xr[i] = nA;
            xr[H + i] = nB;
            dA = nA;
            dB = nB;
            gA = ga;
        }
        aA = tg[2 * (H - 1) + 1];
        if (!lastB) aB = aA;
    }
    // ---- backward sweeps: row 1 of a block in terms of its first and last unknowns
    double br = 0.0, cr = 0.0;
    T rA = zzero<T>(), rB = zzero<T>();
    if (live) {
        const double2 t2 = tab[H - 2];
        br = t2.x;
        cr = t2.y;
        rA = xr[H - 2];
        rB = xr[MT - 2];
#pragma unroll
        for (int i = H - 3; i >= 1; --i) {
            const double g = tg[2 * i];
            rA = zsub(xr[i], zmul(g, rA));
            rB = zsub(xr[H + i], zmul(g, rB));
        }
    }
    // ---- E0 of both blocks (A's first row is the system's row 0 on lane 0) -----------
    const bool first = lane == 0;
    const double a0 = first ? A0 : 1.0, b0 = first ? B0 : lam, c0 = first ? C0 : 1.0;
    const double qA = 1.0 / (b0 - c0 * br);
    const double e0aA = a0 * qA, e0cA = -c0 * cr * qA;
    const T e0dA = zmul(qA, zsub(d0, zmul(c0, rA)));
    const double qB = 1.0 / (lam - br);
    const double e0aB = qB, e0cB = -cr * qB;
    const T e0dB = zmul(qB, zsub(live ? xr[H] : zzero<T>(), rB));
    // ---- rows of the blocks' last unknowns --------------------------------------------
    // l_A:  raA l_B(prev lane) + rbA l_A + rcA l_B = rdA
    const double raA = -aA * e0aA, rbA = 1.0 - aA * e0cA - gA * e0aB, rcA = -gA * e0cB;
    const T rdA = zsub(zsub(dA, zmul(aA, e0dA)), zmul(gA, e0dB));
    // l_B:  raB l_A + rbB l_B + rcB l_A(next lane) = rdB
    const int nxt = (lane + 1) & (P - 1);
    const double na0 = zshfl(e0aA, nxt, P), nc0 = zshfl(e0cA, nxt, P);
    const T nd0 = zshfl(e0dA, nxt, P);
    const double raB = -aB * e0aB, rbB = 1.0 - aB * e0cB - gB * na0, rcB = -gB * nc0;
    const T rdB = zsub(zsub(dB, zmul(aB, e0dB)), zmul(gB, nd0));
    // l_A = pd - pa l_B(prev lane) - pc l_B, substituted into the l_B rows
    const double iA = 1.0 / rbA;
    const double pa = raA * iA, pc = rcA * iA;
    const T pd = zmul(iA, rdA);
    const double npa = zshfl(pa, nxt, P), npc = zshfl(pc, nxt, P);
    const T npd = zshfl(pd, nxt, P);
    const T lB = zsolve_reduced(-raB * pa, rbB - raB * pc - rcB * npa, -rcB * npc,
                                zsub(zsub(rdB, zmul(raB, pd)), zmul(rcB, npd)), lane, P, periodic);
    const T lBp = zshfl(lB, (lane + P - 1) & (P - 1), P);
    const T lA = zsub(zsub(pd, zmul(pa, lBp)), zmul(pc, lB));
    const T fA = zsub(zsub(e0dA, zmul(e0aA, lBp)), zmul(e0cA, lA));
    const T fB = zsub(zsub(e0dB, zmul(e0aB, lA)), zmul(e0cB, lB));
    // ---- recover both blocks' rows ------------------------------------------------------
    if (!live) return;
    if (clear) {
#pragma unroll
        for (int i = 0; i < MT; ++i) xr[i] = zzero<T>();
        return;
    }
    T xa = lA, xb = lB;
    xr[H - 1] = lA;
    xr[MT - 1] = lB;
#pragma unroll
    for (int i = H - 2; i >= 1; --i) {
        const double2 ti = tab[i];
        xa = zsub(zsub(xr[i], zmul(ti.y, fA)), zmul(ti.x, xa));
        xb = zsub(zsub(xr[H + i], zmul(ti.y, fB)), zmul(ti.x, xb));
        xr[i] = xa;
        xr[H + i] = xb;
    }
    xr[0] = fA;
    xr[H] = fB;
}

// shared-memory layout of one CTA
struct ZLayout {
    int pitch;       // tile column pitch (elements)
    int mmax;        // table rows per group
    int groups;      // groups (systems in flight) per CTA
    int P;           // lanes per system
    size_t tile_off, tab_off, red_off, stg_off, bytes;
};

// g32: the FP32 spectrum is first copied into a staging area [k][s] of
// TS x nz FP32 elements behind the rest
PP_HD ZLayout zlayout(int TS, int nz, int P, bool cplx, int nthreads, bool g32 = false)
{
    ZLayout L;
    const size_t e = cplx ? 16 : 8;
    L.P = P;
    L.pitch = zpitch(nz);
    L.mmax = (nz + P - 1) / P + 1;
    L.groups = nthreads / P;
    L.tile_off = 0;
    L.tab_off = (size_t)TS * L.pitch * e;
    L.tab_off = (L.tab_off + 15) & ~(size_t)15;
    // scratch of the pivot-table build: the b_i recurrence of every system
    L.red_off = L.tab_off + (size_t)TS * L.mmax * 16;
    L.bytes = L.red_off + (size_t)TS * L.mmax * 8;
    L.stg_off = (L.bytes + 15) & ~(size_t)15;
    if (g32) L.bytes = L.stg_off + (size_t)TS * nz * (cplx ? 8 : 4);
    return L;
}

template <typename T>
struct ZTo32;
template <>
struct ZTo32<double> {
    using type = float;
    static PP_D double up(float v) { return (double)v; }
    static PP_D float down(double v) { return (float)v; }
};
template <>
struct ZTo32<double2> {
    using type = float2;
    static PP_D double2 up(float2 v) { return make_double2(v.x, v.y); }
    static PP_D float2 down(double2 v) { return make_float2((float)v.x, (float)v.y); }
};
// a stored element (FP64, or FP32 for the refined solve's spectra) to and from
// the FP64 arithmetic type T
template <typename T>
PP_D T zup(T v) { return v; }
template <typename T>
PP_D T zup(typename ZTo32<T>::type v) { return ZTo32<T>::up(v); }
template <typename TG, typename T>
PP_D TG zdown(T v)
{
    if constexpr (std::is_same<TG, T>::value) return v;
    else return ZTo32<T>::down(v);
}

// G32: the spectrum in global memory is FP32 (refined mixed-precision solve);
// all arithmetic stays FP64 (the shared tile too, except in the bulk-copied
// chunks, which hold the stored elements).  MT > 0: every lane keeps its rows
// in registers through the three sweeps, reading and writing its rows of the
// tile once -- exactly MT rows each (CAP = false, nz = P MT, MT = 8, 10, 12, 16, 20, 24, 32),
// or at most MT (CAP = true, MT = 8, 12, 16, 24, 32: M = nz / P or one more,
// the registers indexed statically under i < M guards); MT = 0: any nz, the
// sweeps work on the tile in shared memory.  SPLIT: exactly MT = 10, 12, 16, 20, 24 or 32
// rows per lane, swept as two half blocks (zsolve_split).
template <bool CPLX, bool G32, int MT, bool CAP, bool SPLIT>
PP_D void zsolve_body(PPZArgs a)
{
    using T = typename std::conditional<CPLX, double2, double>::type;
    using T32 = typename ZTo32<T>::type;
    extern __shared__ __align__(16) unsigned char zsm_raw[];
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int P = a.P;
    const ZLayout Lz = zlayout(a.TS, nz, P, CPLX, blockDim.x, G32);
    T* tile = reinterpret_cast<T*>(zsm_raw + Lz.tile_off);

    const int group = threadIdx.x / P;
    const int lane = threadIdx.x - group * P;

    const int ky = blockIdx.x / a.tiles_x;
    const int kx0 = (blockIdx.x - ky * a.tiles_x) * a.TS;
    const int ts = min(a.TS, nx - kx0);
    T* g = reinterpret_cast<T*>(a.data);
    T32* g32 = reinterpret_cast<T32*>(a.data);
    // row k of system s at k * plane + col0 + s: the usual [k][ky][kx] layout,
    // or the z-tiled one, where this CTA's tile is one contiguous block
    const long plane = a.tiled ? (long)a.TS : (long)nx * ny;
    const long col0 = a.tiled ? (long)blockIdx.x * nz * a.TS : (long)ky * nx + kx0;
    // Bulk-copied tiles: z-tiled, rows in registers, and either the split
    // kernels or complex spectra with uneven row counts (where complex uneven
    // rows gained 0.30 -> 0.28 ms at 384^3, real ones lost 3 %).  Each lane
    // block of the tile (the lane's rows x TS systems, contiguous in global
    // memory) moves as one bulk copy (the copy engine, not the LSU pipe) into a
    // chunk of shared memory,
    // the chunks 16 bytes past the longest block so that the lanes of a phase
    // read distinct banks (or two-way shared ones at one system per half
    // warp); the tile goes back the same way.  FP32 spectra (G32) stay FP32 in
    // the chunks: the lanes convert their rows on the way into and out of
    // registers.  Lane L's block is rows L brows + min(L, brem) on, brows + 1
    // of them for the first brem lanes, brows for the rest.
    using TG = typename std::conditional<G32, T32, T>::type;  // element in global memory
    const int brows = SPLIT ? MT : nz / P, brem = SPLIT ? 0 : nz - brows * P;  // split: nz = P MT
    const int crow = a.TS * (int)sizeof(TG);                  // bytes of one tile row
    const int cpitch = (brows + (brem ? 1 : 0)) * crow + 16;
    const bool bulk = (SPLIT || (CAP && CPLX)) && a.tiled && ts == a.TS && crow % 16 == 0 &&
                      (size_t)P * cpitch <= Lz.tab_off && (reinterpret_cast<uintptr_t>(a.data) & 15) == 0;
    __shared__ __align__(8) unsigned long long zbar;
    const unsigned bar = smem_u32(&zbar);
    unsigned char* gtile = G32 ? reinterpret_cast<unsigned char*>(g32 + col0) : reinterpret_cast<unsigned char*>(g + col0);

    // ---- load the tile asynchronously (thread -> (system, row) without division:
    //      TS is a power of two) and build the pivot tables while it lands ------------
    const int lts = __ffs(a.TS) - 1;
    {
        const int s = threadIdx.x & (a.TS - 1);
        const int kstep = blockDim.x >> lts;
        if (s < ts && !bulk) {
            if (G32) {
                // FP32 elements copied asynchronously into the staging area;
                // converted to the FP64 tile once they have landed
                T32* stg = reinterpret_cast<T32*>(zsm_raw + Lz.stg_off);
                for (int k = threadIdx.x >> lts; k < nz; k += kstep) {
                    if (sizeof(T32) == 8) cp_async8(&stg[k * a.TS + s], &g32[k * plane + col0 + s]);
                    else cp_async4(&stg[k * a.TS + s], &g32[k * plane + col0 + s]);
                }
            }
        }
        if (bulk) {
            if (threadIdx.x == 0) {
                mbar_init(bar);
                mbar_expect(bar, (unsigned)(nz * crow));
                for (int c = 0; c < P; ++c)
                    bulk_g2s(zsm_raw + (size_t)c * cpitch, gtile + (size_t)(c * brows + min(c, brem)) * crow,
                             (unsigned)((brows + (c < brem ? 1 : 0)) * crow), bar);
            }
        } else if (!G32)
            zt_each<T>(a.TS, lts, nz, ts, [&](int s2, int k) {
                if (sizeof(T) == 16) cp_async16(&tile[s2 * Lz.pitch + zpos(k)], &g[k * plane + col0 + s2]);
                else cp_async8(&tile[s2 * Lz.pitch + zpos(k)], &g[k * plane + col0 + s2]);
            });
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    // interior pivots of a block, depending only on lambda: with b_0 = 1,
    // b_1 = lambda, b_i = lambda b_{i-1} - b_{i-2} (Chebyshev U_i(lambda/2)),
    //   gamma_i = b_{i-1} / b_i,  alpha_i = (-1)^{i-1} / b_i,
    // the same numbers as the Thomas recurrence gamma_i = 1 / (lambda - gamma_{i-1}).
    // One thread per system; the divisions are independent.  |b_i| grows like
    // |lambda|^i, so where mm log2|lambda| could leave the double range the
    // division recurrence is used instead.
    // Phase 1, one thread per system: b_i by the recurrence (FMAs only) into
    // the scratch bytes, or -- where |b_i| could overflow -- the division
    // recurrence straight into the table, marked by b_0 = 0.
    double* bsc = reinterpret_cast<double*>(zsm_raw + Lz.red_off);
    const int mm = Lz.mmax;
    const int mcount = SPLIT ? MT / 2 : mm;  // entries built (split blocks: MT / 2 rows)
    for (int s = threadIdx.x; s < ts; s += blockDim.x) {
        const double lam = (-2.0 + a.ax[kx0 + s] * a.Cx) + a.ay[ky] * a.Cy;
        double* b = bsc + (size_t)s * mm;
        if ((double)mcount * log2(fabs(lam) + 1.0) < 900.0) {
            double bm = 1.0, bc = lam;
            b[0] = 1.0;
            for (int i = 1; i < mcount; ++i) {
                b[i] = bc;
                const double bn = lam * bc - bm;
                bm = bc;
                bc = bn;
            }
        } else {
            double2* tb = reinterpret_cast<double2*>(zsm_raw + Lz.tab_off) + (size_t)s * mm;
            double gp = 0.0, ap = 0.0;
            for (int i = 1; i < mcount; ++i) {
                const double p = (i == 1) ? 1.0 / lam : 1.0 / (lam - gp);
                const double al = (i == 1) ? p : -ap * p;
                tb[i] = make_double2(p, al);
                gp = p;
                ap = al;
            }
            b[0] = 0.0;
        }
    }
    __syncthreads();
    // Phase 2, every thread: gamma_i = b_{i-1} / b_i, alpha_i = (-1)^{i-1} / b_i,
    // one reciprocal per entry, the entries of all systems spread over the CTA
    {
        // blockDim.x / TS threads per system (both powers of two)
        const int ltp = __ffs(blockDim.x) - 1 - lts;
        const int s = threadIdx.x >> ltp;
        const double* b = bsc + (size_t)s * mm;
        if (s < ts && b[0] != 0.0)
            for (int i = (threadIdx.x & ((1 << ltp) - 1)) + 1; i < mcount; i += 1 << ltp) {
                const double inv = 1.0 / b[i];
                reinterpret_cast<double2*>(zsm_raw + Lz.tab_off)[(size_t)s * mm + i] =
                    make_double2(b[i - 1] * inv, (i & 1) ? inv : -inv);
            }
    }
    cp_async_wait_all();
    if (bulk) {
        // a bounded wait (about a second of polls): a CTA whose copies never
        // land counts itself and leaves without output, with every thread
        const bool landed = mbar_wait0(bar, 1L << 22);
        if (__syncthreads_or(!landed)) {
            if (threadIdx.x == 0 && a.err) atomicAdd(a.err, 1);
            return;
        }
    } else {
        __syncthreads();
    }
    if (G32 && !bulk) {
        const T32* stg = reinterpret_cast<const T32*>(zsm_raw + Lz.stg_off);
        const int s = threadIdx.x & (a.TS - 1);
        const int kstep = blockDim.x >> lts;
        if (s < ts)
            for (int k = threadIdx.x >> lts; k < nz; k += kstep)
                tile[s * Lz.pitch + zpos(k)] = ZTo32<T>::up(stg[k * a.TS + s]);
        __syncthreads();
    }

    const int bsz = nz / P;
    const int rem = nz - bsz * P;
    constexpr bool EXACT = MT > 0 && !CAP;
    const int M = EXACT ? MT : bsz + (lane < rem ? 1 : 0);
    const int s0 = lane * bsz + min(lane, rem);
    const bool periodic = a.zlo == PP_Z_PERIODIC;
    const bool has_d = a.zlo == PP_Z_DIRICHLET || a.zhi == PP_Z_DIRICHLET;
    const unsigned full = 0xffffffffu;

    // all groups of a warp run the same number of iterations (warp-synchronous steps)
    const int ngroups = Lz.groups;
    const int iters = (a.TS + ngroups - 1) / ngroups;
    for (int it = 0; it < iters; ++it) {
        const int s = group + it * ngroups;
        const bool live = s < ts;
        const int kx = kx0 + (live ? s : 0);
        const double lam = (-2.0 + a.ax[kx] * a.Cx) + a.ay[ky] * a.Cy;
        const bool zero = fabs(lam + 2.) < 1.e-10;
        const bool pin = zero && (periodic || a.pin_always || !has_d);
        T* col = tile + (live ? s : 0) * Lz.pitch;
        const double2* tab = reinterpret_cast<const double2*>(zsm_raw + Lz.tab_off) + (size_t)(live ? s : 0) * Lz.mmax;
        // the lane's rows: registers (MT > 0) or the tile column
        // with MT a power of two >= 8 and s0 = lane MT, zpos(s0 + i) = zpos(s0) + zpos(i)
        // (s0 + i never crosses a multiple of 16 that s0 does not); 10, 12, 20
        // and 24 rows index the skewed column directly
        constexpr bool ZP2 = (MT & (MT - 1)) == 0;
        T xr[MT > 0 ? MT : 1];
        T* xcol = col + zpos(s0);
        // (bulk) the lane's rows of system s in its chunk, TS apart
        TG* lrow = reinterpret_cast<TG*>(zsm_raw + (size_t)lane * cpitch) + (live ? s : 0);
        if constexpr (EXACT) {
            if (bulk) {
#pragma unroll
                for (int i = 0; i < MT; ++i) xr[i] = live ? zup<T>(lrow[i * a.TS]) : zzero<T>();
            } else if constexpr (ZP2) {
#pragma unroll
                for (int i = 0; i < MT; ++i) xr[i] = live ? xcol[zpos(i)] : zzero<T>();
            } else {
#pragma unroll
                for (int i = 0; i < MT; ++i) xr[i] = live ? col[zpos(s0 + i)] : zzero<T>();
            }
        } else if constexpr (MT > 0) {
#pragma unroll
            for (int i = 0; i < MT; ++i)
                xr[i] = (live && i < M) ? (bulk ? zup<T>(lrow[i * a.TS]) : col[zpos(s0 + i)]) : zzero<T>();
        }
        auto X = [&](int i) -> T& {
            if constexpr (MT > 0) return xr[i];
            else return col[zpos(s0 + i)];
        };

        double A0, B0, C0, AN, BN, CN;
        if (periodic) {
            A0 = 1.0;
            B0 = pin ? 1.0 : lam;
            C0 = pin ? 0.0 : 1.0;
            AN = 1.0;
            BN = lam;
            CN = 1.0;
        } else {
            A0 = 0.0;
            B0 = pin ? 1.0 : (a.zlo == PP_Z_NEUMANN ? lam + 1. : lam - 1.);
            C0 = pin ? 0.0 : 1.0;
            AN = 1.0;
            BN = a.zhi == PP_Z_NEUMANN ? lam + 1.0 : lam - 1.;
            CN = 0.0;
        }

        if constexpr (SPLIT) {
            static_assert(EXACT, "the split solve keeps exactly MT rows per lane");
            T d0 = zzero<T>();
            if (live) {
                d0 = xr[0];
                if (lane == 0 && periodic && pin) {
                    const T last = bulk ? zup<T>(reinterpret_cast<const TG*>(zsm_raw + (size_t)(P - 1) * cpitch)[(MT - 1) * a.TS + s])
                                        : col[zpos(nz - 1)];
                    d0 = zmul(0.5, zadd(d0, last));
                }
            }
            zsolve_split<MT>(xr, tab, d0, live, zero && a.skip_zero, lane, P, periodic, lam, A0, B0, C0, AN, BN, CN);
        } else {
            // ---- forward sweep of the lane's block -------------------------------------
            // row i (i >= 1) becomes alpha_i x_0 + x_i + gamma_i x_{i+1} = delta_i; delta
            // overwrites the RHS in the tile (only this lane touches these rows)
            double rA0 = 1.0, rB0 = lam, rC0 = 1.0;
            if (s0 == 0) {
                rA0 = A0;
                rB0 = B0;
                rC0 = C0;
            }
            T rD0 = zzero<T>(), dprev = zzero<T>();
            // alpha of the block's last row: the table's, or the system's last row
            double aprev = 0.0, gprev = 0.0;
            bool last_special = false;
            const double* tg = reinterpret_cast<const double*>(tab);  // gamma_i = tg[2i], alpha_i = tg[2i+1]
            if (live) {
                rD0 = X(0);
                // the tile still holds every lane's input here (registers are
                // written back at the end)
                if (s0 == 0 && periodic && pin) {
                    // row nz - 1: the last of lane P - 1's brows rows
                    const T last = bulk ? zup<T>(reinterpret_cast<const TG*>(zsm_raw + (size_t)(P - 1) * cpitch)[(brows - 1) * a.TS + s])
                                        : col[zpos(nz - 1)];
                    rD0 = zmul(0.5, zadd(rD0, last));
                }
#pragma unroll
                for (int i = 1; i < (MT > 0 ? MT : M); ++i) {
                    if (CAP && i >= M) break;
                    const int gk = s0 + i;
                    const T D = X(i);
                    double ga;
                    T dn;
                    // with MT rows per lane only the last unrolled row can be the
                    // system's last row: for real spectra the test is resolved at
                    // compile time elsewhere (for complex ones the register cost of
                    // the specialised code outweighs it).  Interior rows need gamma
                    // only; alpha matters for the block's last row alone.
                    if (!((MT == 0 || CAP || CPLX || i == MT - 1) && gk == nz - 1)) {
                        ga = tg[2 * i];
                        dn = (i == 1) ? zmul(ga, D) : zmul(ga, zsub(D, dprev));
                    } else if (i == 1) {
                        const double inv = 1.0 / BN;
                        aprev = AN * inv;
                        ga = CN * inv;
                        dn = zmul(inv, D);
                        last_special = true;
                    } else {
                        const double p = 1.0 / (BN - AN * gprev);
                        aprev = -AN * tg[2 * (i - 1) + 1] * p;
                        ga = CN * p;
                        dn = zmul(p, zsub(D, zmul(AN, dprev)));
                        last_special = true;
                    }
                    X(i) = dn;
                    gprev = ga;
                    dprev = dn;
                }
                if (!last_special) aprev = tg[2 * (M - 1) + 1];
            }
            // (alpha, gamma, delta) of the block's last row: the reduced row E1
            const double e1a = aprev, e1c = gprev;
            const T e1d = dprev;
            __syncwarp(full);

            // ---- backward sweep: row 1 in terms of x_0 and x_{M-1} ------------------------
            // x_1 = dr - br x_0 - cr x_{M-1}.  The spikes are entries of the inverse
            // of the block's interior matrix tridiag(1, lambda, 1) of order n = M-2:
            // br = [T^-1]_11 = b_{n-1} / b_n = gamma_n and cr = [T^-1]_1n =
            // (-1)^{n+1} / b_n = alpha_n, both in the table; only dr is swept.
            double br = 0, cr = 0;
            T dr = zzero<T>();
            if (live && M >= 3) {
                const double2 t2 = tab[M - 2];
                br = t2.x;
                cr = t2.y;
                const double* tg = reinterpret_cast<const double*>(tab);
                if constexpr (CAP) {
                    // registers indexed statically: rows above M - 2 are skipped
#pragma unroll
                    for (int i = MT - 2; i >= 1; --i) {
                        if (i > M - 2) continue;
                        dr = (i == M - 2) ? X(i) : zsub(X(i), zmul(tg[2 * i], dr));
                    }
                } else {
                    dr = X(M - 2);
#pragma unroll
                    for (int i = M - 3; i >= 1; --i) dr = zsub(X(i), zmul(tg[2 * i], dr));
                }
            }
            double e0a, e0c;
            T e0d;
            if (M == 2) {
                const double inv = 1.0 / rB0;
                e0a = rA0 * inv;
                e0c = rC0 * inv;
                e0d = zmul(inv, rD0);
            } else {
                const double q = 1.0 / (rB0 - rC0 * br);
                e0a = rA0 * q;
                e0c = -rC0 * cr * q;
                e0d = zmul(q, zsub(rD0, zmul(rC0, dr)));
            }

            // ---- reduced system ---------------------------------------------------------------
            // lane L's rows E0: f_L + e0a l_{L-1} + e0c l_L = e0d and
            //                E1: e1a f_L + l_L + e1c f_{L+1} = e1d
            // in its first (f) and last (l) unknowns.  Eliminating every f_L with E0
            // leaves a tridiagonal system in l alone, one row per lane (the Schur
            // complement, diagonally dominant with the original):
            //   -e1a e0a l_{L-1} + (1 - e1a e0c - e1c e0a') l_L - e1c e0c' l_{L+1}
            //       = e1d - e1a e0d - e1c e0d'          (' : lane L+1)
            // The lane indices wrap (periodic z); without it e0a = 0 on the first lane
            // and e1c = 0 on the last, so the wrapped values carry no weight.  It is
            // solved by parallel cyclic reduction over warp shuffles, the periodic one
            // through Sherman-Morrison, and f_L follows from E0.
            const int nxt = (lane + 1) & (P - 1);
            const double na0 = zshfl(e0a, nxt, P), nc0 = zshfl(e0c, nxt, P);
            const T nd0 = zshfl(e0d, nxt, P);
            double ra = -e1a * e0a;
            const double rb = 1.0 - e1a * e0c - e1c * na0;
            double rc = -e1c * nc0;
            T rd = zsub(zsub(e1d, zmul(e1a, e0d)), zmul(e1c, nd0));
            const T xl = zsolve_reduced(ra, rb, rc, rd, lane, P, periodic);
            const T xlp = zshfl(xl, (lane + P - 1) & (P - 1), P);
            const T xf = zsub(zsub(e0d, zmul(e0a, xlp)), zmul(e0c, xl));
            // ---- recover the block's rows ---------------------------------------------------
            if (live && zero && a.skip_zero) {
                // the kx = ky = 0 column is solved separately (in FP64 from plane sums)
#pragma unroll
                for (int i = 0; i < (MT > 0 ? MT : M); ++i) X(i) = zzero<T>();
            } else if (live && CAP) {
                T xn = xl;
#pragma unroll
                for (int i = MT - 1; i >= 1; --i) {
                    if (i > M - 1) continue;
                    if (i == M - 1) {
                        X(i) = xl;
                    } else {
                        const double2 ti = tab[i];
                        xn = zsub(zsub(X(i), zmul(ti.y, xf)), zmul(ti.x, xn));
                        X(i) = xn;
                    }
                }
                X(0) = xf;
            } else if (live) {
                T xn = xl;
                X(M - 1) = xl;
#pragma unroll
                for (int i = M - 2; i >= 1; --i) {
                    const double2 ti = tab[i];
                    xn = zsub(zsub(X(i), zmul(ti.y, xf)), zmul(ti.x, xn));
                    X(i) = xn;
                }
                X(0) = xf;
            }
        }
        if constexpr (EXACT) {
            if (live && bulk) {
#pragma unroll
                for (int i = 0; i < MT; ++i) lrow[i * a.TS] = zdown<TG>(xr[i]);
            } else if (live) {
                if constexpr (ZP2) {
#pragma unroll
                    for (int i = 0; i < MT; ++i) xcol[zpos(i)] = xr[i];
                } else {
#pragma unroll
                    for (int i = 0; i < MT; ++i) col[zpos(s0 + i)] = xr[i];
                }
            }
        } else if constexpr (MT > 0) {
            if (live) {
#pragma unroll
                for (int i = 0; i < MT; ++i) {
                    if (i >= M) continue;
                    if (bulk) lrow[i * a.TS] = zdown<TG>(xr[i]);
                    else col[zpos(s0 + i)] = xr[i];
                }
            }
        }
        __syncwarp(full);
    }
    if (bulk) fence_proxy_async_smem();  // the rows written above, read by the bulk copies
    __syncthreads();

    if (bulk) {
        if (threadIdx.x == 0) {
            for (int c = 0; c < P; ++c)
                bulk_s2g(gtile + (size_t)(c * brows + min(c, brem)) * crow, zsm_raw + (size_t)c * cpitch,
                         (unsigned)((brows + (c < brem ? 1 : 0)) * crow));
            bulk_commit_wait_read();
        }
    } else if (G32) {
        const int s = threadIdx.x & (a.TS - 1);
        const int kstep = blockDim.x >> lts;
        if (s < ts)
            for (int k = threadIdx.x >> lts; k < nz; k += kstep)
                g32[k * plane + col0 + s] = ZTo32<T>::down(tile[s * Lz.pitch + zpos(k)]);
    } else
        zt_each<T>(a.TS, lts, nz, ts, [&](int s2, int k) { g[k * plane + col0 + s2] = tile[s2 * Lz.pitch + zpos(k)]; });
}


template <bool CPLX, bool G32, int MT, bool CAP, bool SPLIT>
__global__ void __launch_bounds__(PP_Z_THREADS) zsolve_kernel(PPZArgs a)
{
    zsolve_body<CPLX, G32, MT, CAP, SPLIT>(a);
}
// The split kernels held to 128 registers (two CTAs of 256 threads, or four
// of 128, per SM): their sweeps are bound by the latency of dependent FP64
// operations, and the extra resident warps outweigh a few spilled values
// (512^3: real 32 rows per lane 0.436 -> 0.380 ms with 92 bytes spilled,
// complex 16 rows 0.446 -> 0.381 ms; FP32 complex spectra 0.37 -> 0.33 ms).
// Not for FP32 real spectra, whose conversions make the cap cost more than
// it gains (0.33 -> 0.36 ms).  A separate kernel: naming a minimum of one
// CTA per SM in the other kernels' launch bounds lets the compiler spend
// more registers on them than the one-argument form does.
template <bool CPLX, bool G32, int MT>
__global__ void __launch_bounds__(PP_Z_THREADS, 2) zsolve_split_r128_kernel(PPZArgs a)
{
    zsolve_body<CPLX, G32, MT, false, true>(a);
}
// the split kernel a launch takes (only that one is compiled)
template <bool CPLX, bool G32, int MT>
void (*split_kernel())(PPZArgs)
{
    if constexpr (CPLX || !G32) return zsolve_split_r128_kernel<CPLX, G32, MT>;
    else return zsolve_kernel<CPLX, G32, MT, false, true>;
}
}  // namespace

int pp_zsolve_lanes(int nz, bool cplx, bool large)
{
    // about 32 rows per lane (16 for complex data, whose tile is twice as
    // large, so that a CTA still keeps every group busy).  Grids with many
    // systems (large) take the fewest lanes that leave at most that many rows,
    // so that any nz keeps its rows in registers; smaller grids keep more
    // resident CTAs with the shared-memory rows (batches of small grids run
    // concurrently, where occupancy counts more)
    const int rows = cplx ? 16 : 32;
    int P = 1;
    if (large)
        while (P < 32 && (nz + P - 1) / P > rows) P *= 2;
    else
        while (P < 32 && 2 * P <= nz / rows) P *= 2;
    while (P > 1 && P > nz / 2) P /= 2;
    return P;
}

bool pp_zsolve_large(long systems) { return systems >= PP_Z_LARGE_SYSTEMS; }

// launch shape: systems per CTA (one lane group each) and threads per CTA,
// keeping the CTA within ~56 KB of shared memory so about four fit on an SM
void pp_zsolve_config(int nz, bool cplx, int nx, int* TS, int* threads)
{
    const int P = pp_zsolve_lanes(nz, cplx, false);
    int ts = PP_Z_THREADS / P;
    auto bytes = [&](int t) {
        const int th = t * P < 32 ? 32 : t * P;
        return zlayout(t, nz, P, cplx, th).bytes;
    };
    while (ts > 1 && bytes(ts) > 56 * 1024) ts >>= 1;
    while (ts > 1 && ts > nx) ts >>= 1;
    *TS = ts;
    *threads = ts * P < 32 ? 32 : ts * P;
}

// a lane count the kernel accepts: a power of two <= 32 leaving every lane at
// least two rows
int pp_zsolve_valid_lanes(int nz, int P)
{
    return P >= 1 && P <= 32 && (P & (P - 1)) == 0 && (P == 1 || P <= nz / 2);
}

size_t pp_zsolve_smem_p(int TS, int nz, bool cplx, int P)
{
    const int th = TS * P < 32 ? 32 : TS * P;
    return zlayout(TS, nz, P, cplx, th).bytes;
}

// the launch shape for a chosen lane count (0 or invalid: the default) and
// systems per CTA (0: as many as fit ~56 KB of shared memory)
void pp_zsolve_config_p(int nz, bool cplx, int nx, int lanes, int* TS, int* threads, int systems, int ny)
{
    const int P = pp_zsolve_valid_lanes(nz, lanes) ? lanes : pp_zsolve_lanes(nz, cplx, pp_zsolve_large((long)nx * ny));
    int ts = PP_Z_THREADS / P;
    if (systems >= 1 && (systems & (systems - 1)) == 0 && systems <= ts) {
        ts = systems;
        while (ts > 1 && pp_zsolve_smem_p(ts, nz, cplx, P) > 200 * 1024) ts >>= 1;
    }
    while (ts > 1 && systems == 0 && pp_zsolve_smem_p(ts, nz, cplx, P) > 56 * 1024) ts >>= 1;
    while (ts > 1 && ts > nx) ts >>= 1;
    *TS = ts;
    *threads = ts * P < 32 ? 32 : ts * P;
}

int pp_zsolve_max_nz(bool cplx, bool g32)
{
    int lo = 3, hi = 1 << 16;  // lo fits, hi does not
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (zlayout(1, mid, 32, cplx, 32, g32).bytes <= (size_t)227 * 1024) lo = mid;
        else hi = mid;
    }
    return lo;
}

cudaError_t pp_launch_zsolve(const PPZArgs& a0, bool cplx, cudaStream_t st)
{
    if (a0.nz < 3 || a0.nz > pp_zsolve_max_nz(cplx, a0.data_fp32 != 0)) return cudaErrorInvalidValue;
    PPZArgs a = a0;
    const bool large = pp_zsolve_large((long)a.nx * a.ny);
    if (!pp_zsolve_valid_lanes(a.nz, a.P)) a.P = pp_zsolve_lanes(a.nz, cplx, large);
    const int threads = a.TS * a.P < 32 ? 32 : a.TS * a.P;
    if (threads > PP_Z_THREADS) return cudaErrorInvalidValue;
    const size_t smem = zlayout(a.TS, a.nz, a.P, cplx, threads, a.data_fp32 != 0).bytes;
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    dim3 grid(a.ny * a.tiles_x), block(threads);
    cudaError_t e;
    // rows per lane fixed at compile time where every lane has the same count;
    // else the smallest register capacity that holds every lane's rows
    const int rows = a.nz / a.P, rmax = (a.nz + a.P - 1) / a.P;
    const int mt = (a.nz % a.P == 0 && (rows == 8 || rows == 16 || ((rows == 10 || rows == 12) && cplx) ||
                                        ((rows == 20 || rows == 24 || rows == 32) && !cplx))) ? rows : 0;
    int cap = 0;
    if (!mt && large) {
        if (cplx) cap = rmax <= 8 ? 8 : rmax <= 12 ? 12 : rmax <= 16 ? 16 : 0;
        else cap = rmax <= 8 ? 8 : rmax <= 16 ? 16 : rmax <= 24 ? 24 : rmax <= 32 ? 32 : 0;
    }
#define PP_ZL(C, G, M, K) PP_ZLF((zsolve_kernel<C, G, M, K, false>))
#define PP_ZLK(C, G, M, K, S)                                                                                   \
    do {                                                                                                        \
        PP_ZLF((split_kernel<C, G, M>()));                                                                     \
    } while (0)
#define PP_ZLF(KFN)                                                                                             \
    do {                                                                                                        \
        auto kfn = KFN;                                                                                         \
        if ((e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) \
            return e;                                                                                           \
        kfn<<<grid, block, smem, st>>>(a);                                                                      \
    } while (0)
// (the row counts a complex or real launch never takes are replaced by ones
// it does, so that no dead instance is compiled)
#define PP_ZLM(C, G)                                  \
    do {                                              \
        if (mt == 8) PP_ZL(C, G, 8, false);           \
        else if (mt == 16) PP_ZLK(C, G, 16, false, true); \
        else if (mt == 32 && !C) PP_ZLK(C, G, (C ? 16 : 32), false, true); \
        else if (mt == 24 && !C) PP_ZLK(C, G, (C ? 16 : 24), false, true); \
        else if (mt == 12 && C) PP_ZLK(C, G, (C ? 12 : 16), false, true); \
        else if (mt == 20 && !C) PP_ZLK(C, G, (C ? 16 : 20), false, true); \
        else if (mt == 10 && C) PP_ZLK(C, G, (C ? 10 : 16), false, true); \
        else if (cap == 8) PP_ZL(C, G, 8, true);      \
        else if (cap == 12 && C) PP_ZL(C, G, (C ? 12 : 16), true); \
        else if (cap == 16) PP_ZL(C, G, 16, true);    \
        else if (cap == 24 && !C) PP_ZL(C, G, (C ? 16 : 24), true); \
        else if (cap == 32 && !C) PP_ZL(C, G, (C ? 16 : 32), true); \
        else PP_ZL(C, G, 0, false);                   \
    } while (0)
    if (cplx && a.data_fp32) PP_ZLM(true, true);
    else if (cplx) PP_ZLM(true, false);
    else if (a.data_fp32) PP_ZLM(false, true);
    else PP_ZLM(false, false);
#undef PP_ZLM
#undef PP_ZL
#undef PP_ZLK
#undef PP_ZLF
    return cudaGetLastError();
}
