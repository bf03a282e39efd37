// Shared device helpers for the PittPack B200 solver.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define PP_HD __host__ __device__ __forceinline__
#define PP_D __device__ __forceinline__

// transform kind of one direction (x or y).  The first three are the
// reference's tags (extractTag, src/pencilDcmp.cpp:3636-3668: DST 0, DCT 1,
// FFT 2); the N-D and D-N families are not in the reference.
enum PPKind : int {
    PP_KIND_DST2 = 0,  // D-D: DST-II forward, DST-III inverse
    PP_KIND_DCT2 = 1,  // N-N: DCT-II forward, DCT-III inverse
    PP_KIND_FFT = 2,   // P-P: complex DFT
    PP_KIND_DCT4 = 3,  // N-D: DCT-IV both ways
    PP_KIND_DST4 = 4,  // D-N: DST-IV both ways
};

PP_HD bool pp_kind_is_fft(int k) { return k == PP_KIND_FFT; }
PP_HD bool pp_kind_is_quarter(int k) { return k == PP_KIND_DCT4 || k == PP_KIND_DST4; }

PP_D double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
PP_D double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
PP_D double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
PP_D double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
PP_D double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// multiply by i*s (s = +1 or -1)
PP_D double2 cmul_i(double2 a, double s) { return make_double2(-s * a.y, s * a.x); }

// ---- complex helpers for float2 / double2 ------------------------------------
template <typename C>
struct CReal;
template <>
struct CReal<double2> {
    using type = double;
};
template <>
struct CReal<float2> {
    using type = float;
};

template <typename C>
PP_D C mkc(typename CReal<C>::type x, typename CReal<C>::type y)
{
    C r;
    r.x = x;
    r.y = y;
    return r;
}
template <typename C>
PP_D C c_add(C a, C b) { return mkc<C>(a.x + b.x, a.y + b.y); }
template <typename C>
PP_D C c_sub(C a, C b) { return mkc<C>(a.x - b.x, a.y - b.y); }
template <typename C>
PP_D C c_mul(C a, C b) { return mkc<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <typename C>
PP_D C c_scale(C a, typename CReal<C>::type s) { return mkc<C>(a.x * s, a.y * s); }
// multiply by SIGN * i
template <int SIGN, typename C>
PP_D C c_mul_si(C a) { return SIGN > 0 ? mkc<C>(-a.y, a.x) : mkc<C>(a.y, -a.x); }

// ---- bulk-copy staging (the copy engine, not the LSU pipe) --------------------------
PP_D unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// mbarrier with one arrival, armed for 'bytes' of bulk copies
PP_D void mbar_init(unsigned bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
PP_D void mbar_expect(unsigned bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
// global -> shared bulk copy (both addresses 16-byte aligned, bytes a
// multiple of 16), completion counted on the mbarrier
PP_D void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
// wait for phase 0 of the mbarrier, at most 'limit' polls; true if it completed
PP_D bool mbar_wait0(unsigned bar, long limit)
{
    for (long i = 0; i < limit; ++i) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(bar)
            : "memory");
        if (done) return true;
    }
    return false;
}

// shared -> global bulk copy (both addresses 16-byte aligned, bytes a
// multiple of 16) in the thread's bulk async-group
PP_D void bulk_s2g(void* dst, const void* src, unsigned bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(dst), "r"(smem_u32(src)),
                 "r"(bytes)
                 : "memory");
}
// close the thread's bulk async-group and wait until its copies have read
// their shared-memory sources (the writes to global memory complete on their own)
PP_D void bulk_commit_wait_read()
{
    asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
    asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
}
// this thread's shared-memory writes made visible to later bulk copies
PP_D void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
