// Split-precision analysis contraction on the tcgen05 tensor cores (sm_100a).
//
// The analysis contraction of one scale (s2dw_core_mod.f90:625-673),
//
//   T^k(m, m', +-n) = sum_{l in (bl_lo, bl)} f^k(l, m) * v(l; m', m, n) * (+-1)^l,
//   v(l; m', m, n)  = d^l_{m'm}(pi/2) d^l_{m'n}(pi/2) K_j(l) s(l, n),
//
// is, for a batch of maps k sharing (B, N, alpha, J), a GEMM over l whose
// left operand v does not depend on the map: rows (m', n, l parity) for one
// m, columns (k, re/im); the even-l and odd-l sums E, O give T(+n) = E + O
// and T(-n) = E - O in the epilogue.  Each CTA owns one m, CH consecutive m' ("chains") and
// up to 32 maps.  Per chunk of 32 values of l:
//
//   * one or two walker warps advance the FP64 l-recurrence of d^l_{m'm}
//     (one chain per lane, the recurrence of the FP64 kernel) and write the
//     true-scale values v to shared memory;
//   * all threads cut every value into 6 byte digits of a 48-bit fixed-point
//     integer with a per-row power-of-two scale (two's complement bytes: five
//     unsigned digits and a signed top digit) and store them in the K-major
//     no-swizzle operand layout;
//   * the map operand (f^k(l, m), cut the same way by fdig_kernel, one scale
//     per (m, k, re/im) column) arrives by a bulk copy;
//   * one thread issues 26 tcgen05.mma.kind::i8 (M=128, N=64, K=32): the
//     digit products of significance level t = (5-i)+(5-j) <= 6, each level
//     into its own int32 TMEM accumulator, so every product is summed exactly.
//
// The epilogue reads the seven level accumulators, combines them in FP64 with
// the row and column scales, and applies the +-n phases and the gamma DFT of
// the FP64 kernel (s2dw_core_mod.f90:679-705), writing Tg^k(g, m, m').
//
// The per-row scales come from dexp_kernel, a pre-pass that runs the same
// walker and records the exponent of max_l |v|: the digits of every row then
// use its full 48 bits.  The dropped products (levels 7..10) and the digit
// truncation leave a relative error of ~1e-14 of max|T| (~1e-11 of max|w|
// per scale at bl = 1024).
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>

#include "s2dw_internal.h"

namespace s2dw {
namespace split {

constexpr int MAPS = 32;            // maps per CTA (N = 64 columns: re, im)
constexpr int COLS = 2 * MAPS;
constexpr int ROWS = 128;           // M
constexpr int DIG = 6;              // byte digits per operand
constexpr int LEV = 7;              // significance levels kept
constexpr int KC = 32;              // l per chunk: one K step of kind::i8
constexpr int FIX = 8 * DIG - 1;    // digits hold rint(x * 2^(FIX - E)), |x| < 2^E
// T = 2^(Ed + Ef - SHIFT) * sum_t C_t 2^(-8t)
constexpr int SHIFT = 2 * FIX - 16 * (DIG - 1);
constexpr int A_TILE = ROWS * KC;   // bytes per digit of the v operand
constexpr int B_TILE = COLS * KC;   // bytes per digit of the map operand
constexpr int TMEM_COLS = 512;
constexpr int E_ZERO = -32000;      // exponent of an all-zero row or column
constexpr int E_MIN = -960;         // rows or columns below 2^E_MIN count as zero
constexpr int THREADS = 128;

// Chains per CTA: 2*NP rows per chain (n and l parity), 128 rows, chains a multiple
// of 16 so that every staged table row starts on a 128-byte boundary.
__host__ __device__ constexpr int chains(int NP) { return NP == 1 ? 64 : (NP == 2 ? 32 : 16); }

__device__ __forceinline__ double2 c_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 c_mul(double2 a, double2 b)
{
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// z * i^k
__device__ __forceinline__ double2 c_ipow(double2 z, int k)
{
    switch (k & 3) {
    case 0: return z;
    case 1: return make_double2(-z.y, z.x);
    case 2: return make_double2(-z.x, -z.y);
    default: return make_double2(z.y, -z.x);
    }
}
__device__ __forceinline__ double wmax(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int wmax_i(int v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// ---------------------------------------------------------------------------
// The l-walk of one chain (m', m): the recurrence of lwalk_kernel, in the same
// arithmetic order, so that dexp_kernel and split_kernel see identical values.
// Kw is warp-uniform (the scaled domain of chains whose start underflows).
// ---------------------------------------------------------------------------
struct Chain {
    double e, ep, st, sc;  // sc = 2^-Kw (0 when below the double range)
    int l0, Kw;
};

// 2^E for E in [-1022, 1023], built from the exponent bits.
__device__ __forceinline__ double pow2i(int E) { return __longlong_as_double((long long)(E + 1023) << 52); }
__device__ __forceinline__ double pow2_or_zero(int E) { return E >= -1022 ? pow2i(E) : 0.0; }

// All 32 lanes of the warp call this (lanes without a chain pass valid=false).
__device__ __forceinline__ Chain chain_init(const int32_t *Ste, const double *Stm, int B, int m, int mp, bool valid)
{
    Chain c;
    c.e = 0.0;
    c.ep = 0.0;
    c.st = 0.0;
    c.l0 = valid ? max(mp, m) : INT_MAX;
    int maxe = valid ? (int)Ste[(size_t)max(mp, m) * B + min(mp, m)] : INT_MIN;
    maxe = wmax_i(maxe);
    c.Kw = (maxe != INT_MIN && maxe < S2DW_SCALE_EXP) ? -maxe : 0;
    c.sc = pow2_or_zero(-c.Kw);
    if (valid) {
        const size_t o = (size_t)c.l0 * B + min(mp, m);
        double v = ldexp(Stm[o], (int)Ste[o] + c.Kw);
        if (mp >= m && ((mp - m) & 1)) v = -v;
        c.st = v;
    }
    return c;
}

// Value w(l) = d^l_{m'm} / Om_l(m') (true scale) at row l, then one step to
// l+1.  am = a_m(l), ap = a_{m'}(l), om = Om_l(m).  Values below 2^-1022
// times the walk's scale flush to zero (they are below 2^-600 of the row).
__device__ __forceinline__ double chain_step(Chain &c, int l, double am, double ap, double om)
{
    if (l == c.l0) c.e = c.st;
    const double w = (c.e * om) * c.sc;
    const double en = fma(-(am * ap), c.e, -c.ep);
    c.ep = c.e;
    c.e = en;
    return w;
}

// Called by all lanes after the step of row l when (l & 15) == 15.
__device__ __forceinline__ void chain_renorm(Chain &c)
{
    if (c.Kw > 0) {
        const double mx = wmax(fmax(fabs(c.e), fabs(c.ep)));
        if (mx > pow2i(S2DW_RENORM_EXP)) {
            const int R = min(S2DW_RENORM_EXP, c.Kw);
            const double f = pow2i(-R);
            c.e *= f;
            c.ep *= f;
            c.Kw -= R;
            c.sc = pow2_or_zero(-c.Kw);
        }
    }
}

// ---------------------------------------------------------------------------
// Fixed-point digits
// ---------------------------------------------------------------------------
__device__ __forceinline__ double digit_factor(int E) { return E > E_MIN ? pow2i(FIX - E) : 0.0; }

__device__ __forceinline__ long long to_fixed(double x, double factor)
{
    long long X = __double2ll_rn(x * factor);
    const long long lim = 1LL << FIX;
    X = X > lim - 1 ? lim - 1 : X;
    X = X < -lim ? -lim : X;
    return X;
}

// The DIG digit words of four fixed-point integers: o[d] holds byte d of
// X[0..3] in bytes 0..3.  A 4 x 4 byte transpose of the low words gives
// digits 0-3 and a 4 x 2 one of the high words digits 4-5 (12 byte permutes).
__device__ __forceinline__ void digits4(const long long *X, uint32_t (&o)[DIG])
{
    static_assert(DIG == 6, "six byte digits");
    const uint32_t w0 = (uint32_t)X[0], w1 = (uint32_t)X[1], w2 = (uint32_t)X[2], w3 = (uint32_t)X[3];
    const uint32_t a = __byte_perm(w0, w1, 0x5140), b = __byte_perm(w2, w3, 0x5140);  // bytes 0, 1
    const uint32_t c = __byte_perm(w0, w1, 0x7362), e = __byte_perm(w2, w3, 0x7362);  // bytes 2, 3
    o[0] = __byte_perm(a, b, 0x5410);
    o[1] = __byte_perm(a, b, 0x7632);
    o[2] = __byte_perm(c, e, 0x5410);
    o[3] = __byte_perm(c, e, 0x7632);
    const uint32_t h0 = (uint32_t)(X[0] >> 32), h1 = (uint32_t)(X[1] >> 32), h2 = (uint32_t)(X[2] >> 32),
                   h3 = (uint32_t)(X[3] >> 32);
    const uint32_t f = __byte_perm(h0, h1, 0x5140), g = __byte_perm(h2, h3, 0x5140);  // bytes 4, 5
    o[4] = __byte_perm(f, g, 0x5410);
    o[5] = __byte_perm(f, g, 0x7632);
}

// 16 consecutive K values of one operand row -> the 16-byte K-half of each of
// the DIG digit tiles.  `base` is the row's K-half inside digit tile 0;
// consecutive digit tiles are `tile` bytes apart.
__device__ __forceinline__ void store_digits(unsigned char *base, int tile, const long long *X)
{
    uint32_t o0[DIG], o1[DIG], o2[DIG], o3[DIG];
    digits4(X + 0, o0);
    digits4(X + 4, o1);
    digits4(X + 8, o2);
    digits4(X + 12, o3);
#pragma unroll
    for (int d = 0; d < DIG; d++) *reinterpret_cast<uint4 *>(base + d * tile) = make_uint4(o0[d], o1[d], o2[d], o3[d]);
}

// As store_digits, split by the parity of the K index: row `even` gets the
// values at even K positions (odd ones zero), row `odd` the others.  Byte j
// of each digit word is K position 4w + j, so the parity masks are per byte.
__device__ __forceinline__ void store_digits_parity(unsigned char *even, unsigned char *odd, int tile,
                                                    const long long *X)
{
    uint32_t o0[DIG], o1[DIG], o2[DIG], o3[DIG];
    digits4(X + 0, o0);
    digits4(X + 4, o1);
    digits4(X + 8, o2);
    digits4(X + 12, o3);
    constexpr uint32_t ME = 0x00FF00FFu, MO = 0xFF00FF00u;
#pragma unroll
    for (int d = 0; d < DIG; d++) {
        *reinterpret_cast<uint4 *>(even + d * tile) = make_uint4(o0[d] & ME, o1[d] & ME, o2[d] & ME, o3[d] & ME);
        *reinterpret_cast<uint4 *>(odd + d * tile) = make_uint4(o0[d] & MO, o1[d] & MO, o2[d] & MO, o3[d] & MO);
    }
}

// Offset of (row r, K-half kh) in a K-major no-swizzle tile of R rows x 32
// bytes: 8-row core matrices of 128 contiguous bytes (SBO = 128), the two
// 16-byte K halves R*16 bytes apart (LBO).
__host__ __device__ constexpr int tile_off(int R, int r, int kh) { return kh * R * 16 + (r >> 3) * 128 + (r & 7) * 16; }

// ---------------------------------------------------------------------------
// PTX wrappers: mbarrier, bulk copy, tcgen05
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Waits for the phase with `parity` to complete; gives up after `limit_ns`.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, unsigned long long limit_ns)
{
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = gtimer();
    while (true) {
        if (mbar_try(bar, parity)) return true;
        if (gtimer() - t0 > limit_ns) return false;
    }
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// K-major, no-swizzle shared-memory matrix descriptor (sm_100 format:
// start >> 4 in bits 0-13, LBO >> 4 in 16-29, SBO >> 4 in 32-45, version 1 in
// 46-47, base offset 0, layout type 0 = no swizzle in 61-63).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::i8: S32 accumulator (bits 4-5 = 2), A and B
// format (bits 7-9, 10-12: 0 = u8, 1 = s8), both K-major, N >> 3 in bits
// 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t idesc_i8(int a_signed, int b_signed, int M, int N)
{
    return (2u << 4) | ((uint32_t)a_signed << 7) | ((uint32_t)b_signed << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate)
{
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}
// The seven level accumulators of 16 columns: seven loads, one wait.
__device__ __forceinline__ void tmem_ld16x7(uint32_t taddr, int32_t (&r)[7][16])
{
    static_assert(LEV == 7 && COLS == 64, "level layout");
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%112];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%113];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47}, [%114];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%115];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%64, %65, %66, %67, %68, %69, %70, %71, %72, %73, %74, %75, %76, %77, %78, %79}, [%116];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%80, %81, %82, %83, %84, %85, %86, %87, %88, %89, %90, %91, %92, %93, %94, %95}, [%117];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%96, %97, %98, %99, %100, %101, %102, %103, %104, %105, %106, %107, %108, %109, %110, %111}, [%118];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0][0]), "=r"(r[0][1]), "=r"(r[0][2]), "=r"(r[0][3]), "=r"(r[0][4]), "=r"(r[0][5]), "=r"(r[0][6]), "=r"(r[0][7]), "=r"(r[0][8]), "=r"(r[0][9]), "=r"(r[0][10]), "=r"(r[0][11]), "=r"(r[0][12]), "=r"(r[0][13]), "=r"(r[0][14]), "=r"(r[0][15]),
          "=r"(r[1][0]), "=r"(r[1][1]), "=r"(r[1][2]), "=r"(r[1][3]), "=r"(r[1][4]), "=r"(r[1][5]), "=r"(r[1][6]), "=r"(r[1][7]), "=r"(r[1][8]), "=r"(r[1][9]), "=r"(r[1][10]), "=r"(r[1][11]), "=r"(r[1][12]), "=r"(r[1][13]), "=r"(r[1][14]), "=r"(r[1][15]),
          "=r"(r[2][0]), "=r"(r[2][1]), "=r"(r[2][2]), "=r"(r[2][3]), "=r"(r[2][4]), "=r"(r[2][5]), "=r"(r[2][6]), "=r"(r[2][7]), "=r"(r[2][8]), "=r"(r[2][9]), "=r"(r[2][10]), "=r"(r[2][11]), "=r"(r[2][12]), "=r"(r[2][13]), "=r"(r[2][14]), "=r"(r[2][15]),
          "=r"(r[3][0]), "=r"(r[3][1]), "=r"(r[3][2]), "=r"(r[3][3]), "=r"(r[3][4]), "=r"(r[3][5]), "=r"(r[3][6]), "=r"(r[3][7]), "=r"(r[3][8]), "=r"(r[3][9]), "=r"(r[3][10]), "=r"(r[3][11]), "=r"(r[3][12]), "=r"(r[3][13]), "=r"(r[3][14]), "=r"(r[3][15]),
          "=r"(r[4][0]), "=r"(r[4][1]), "=r"(r[4][2]), "=r"(r[4][3]), "=r"(r[4][4]), "=r"(r[4][5]), "=r"(r[4][6]), "=r"(r[4][7]), "=r"(r[4][8]), "=r"(r[4][9]), "=r"(r[4][10]), "=r"(r[4][11]), "=r"(r[4][12]), "=r"(r[4][13]), "=r"(r[4][14]), "=r"(r[4][15]),
          "=r"(r[5][0]), "=r"(r[5][1]), "=r"(r[5][2]), "=r"(r[5][3]), "=r"(r[5][4]), "=r"(r[5][5]), "=r"(r[5][6]), "=r"(r[5][7]), "=r"(r[5][8]), "=r"(r[5][9]), "=r"(r[5][10]), "=r"(r[5][11]), "=r"(r[5][12]), "=r"(r[5][13]), "=r"(r[5][14]), "=r"(r[5][15]),
          "=r"(r[6][0]), "=r"(r[6][1]), "=r"(r[6][2]), "=r"(r[6][3]), "=r"(r[6][4]), "=r"(r[6][5]), "=r"(r[6][6]), "=r"(r[6][7]), "=r"(r[6][8]), "=r"(r[6][9]), "=r"(r[6][10]), "=r"(r[6][11]), "=r"(r[6][12]), "=r"(r[6][13]), "=r"(r[6][14]), "=r"(r[6][15])
        : "r"(taddr), "r"(taddr + 64), "r"(taddr + 128), "r"(taddr + 192), "r"(taddr + 256), "r"(taddr + 320),
          "r"(taddr + 384)
        : "memory");
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem)), "l"(gmem));
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(smem)), "l"(gmem));
}
__device__ __forceinline__ void cp_commit_all() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// After a wait gave up, the issuer waits for its own bulk copies and MMAs
// still in flight before the CTA tears down (shared memory reuse, TMEM
// deallocation); those complete in microseconds, this bounds the wait.
constexpr unsigned long long DRAIN_NS = 100000000ull;  // 100 ms
// Bounded wait that ignores the abort flag (the drain after an abort).
__device__ __forceinline__ void drain_wait(uint32_t bar, uint32_t parity)
{
    if (mbar_try(bar, parity)) return;
    const unsigned long long t0 = gtimer();
    while (!mbar_try(bar, parity) && gtimer() - t0 <= DRAIN_NS) {
    }
}

// ---------------------------------------------------------------------------
// dexp_kernel: exponent of max_{l in (blo, bl)} |v(l; m', m, n_q)| per
// (m, m', q).  One CTA per (m, chain tile), one lane per chain.
// ---------------------------------------------------------------------------
template <int NP>
__global__ void __launch_bounds__(64) dexp_kernel(SplitArgs a)
{
    constexpr int CH = chains(NP);
    const int2 tile = a.tiles[blockIdx.x];
    const int m = tile.x, p0 = tile.y * CH;
    const int ch = threadIdx.x, mp = p0 + ch;
    const bool valid = ch < CH && mp < a.bl;
    Chain c = chain_init(a.Ste, a.Stm, a.B, m, mp, valid);
    double mx[NP];
#pragma unroll
    for (int q = 0; q < NP; q++) mx[q] = 0.0;
    const int lw = max(m, p0);
    const int mpc = min(mp, a.Bp - 1);
#pragma unroll 4
    for (int l = lw; l < a.bl; l++) {
        const double am = a.Acoef[(size_t)l * a.Bp + m], ap = a.Acoef[(size_t)l * a.Bp + mpc];
        const double om = a.Om[(size_t)l * a.Bp + m];
        const double w = chain_step(c, l, am, ap, om);
        if (l > a.blo && valid) {
#pragma unroll
            for (int q = 0; q < NP; q++) {
                const double v = w * a.G[((size_t)(l - a.blo - 1) * NP + q) * a.Gs + mp];
                mx[q] = fmax(mx[q], fabs(v));
            }
        }
        if ((l & 15) == 15) chain_renorm(c);
    }
    if (valid) {
#pragma unroll
        for (int q = 0; q < NP; q++)
            a.dexp[((size_t)m * a.bl + mp) * NP + q] = (int16_t)(mx[q] > 0.0 ? ilogb(mx[q]) + 1 : E_ZERO);
    }
}

// ---------------------------------------------------------------------------
// fdig_kernel: digits of the map operand for one scale.  One CTA per m;
// column col = 2k + (0: re, 1: im).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(THREADS) fdig_kernel(FdigArgs a)
{
    __shared__ int sE[COLS];
    const int m = blockIdx.x, t = threadIdx.x;
    const int col = t >> 1, half = t & 1, k = col >> 1, comp = col & 1;
    const int lbeg = max(a.blo + 1, m);
    const double *f = reinterpret_cast<const double *>(a.flm) + (size_t)k * a.B * a.B * 2 + (size_t)a.B * m * 2 + comp;
    double mx = 0.0;
    if (k < a.nmaps)
        for (int l = lbeg + ((lbeg & 1) ^ half); l < a.bl; l += 2) mx = fmax(mx, fabs(f[2 * (size_t)l]));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
    const int E = mx > 0.0 ? ilogb(mx) + 1 : E_ZERO;
    if (half == 0) {
        sE[col] = E;
        a.fexp[(size_t)m * COLS + col] = E;
    }
    __syncthreads();
    const double factor = digit_factor(sE[col]);
    const int kh = half;
    for (int ci = 0; ci < a.nch; ci++) {
        const int lb = (a.c0 + ci) * KC + 16 * kh;
        long long X[16];
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const int l = lb + i;
            const double v = (k < a.nmaps && l >= lbeg && l < a.bl) ? f[2 * (size_t)l] : 0.0;
            X[i] = to_fixed(v, factor);
        }
        unsigned char *dst = a.fdig + ((size_t)m * a.nch + ci) * DIG * B_TILE + tile_off(COLS, col, kh);
        store_digits(dst, B_TILE, X);
    }
}

// ---------------------------------------------------------------------------
// split_kernel
// ---------------------------------------------------------------------------
// Thread roles of split_kernel (256 threads, 8 warps):
//   walker warps 0 .. NWALK-1 (one lane per chain) advance the FP64
//     recurrence, one 32-row chunk ahead of the cutters;
//   cutter warps NWALK .. 6 multiply by the factor table and cut digits;
//   warp 7, lane 0 (the issuer) copies the map digits and issues the MMAs.
// They hand chunks over through mbarriers: VFULL (chain values written),
// CUT (digits written, chain values read), done (MMAs finished, tcgen05
// commit), full (map digits landed, bulk-copy transaction count).  Every wait
// is bounded; after a timeout every role skips its remaining work but keeps
// its barrier sequence, so the CTA always reaches the end.
constexpr int SPLIT_THREADS = 256;
constexpr int ISSUER_WARP = 7;

template <int NP>
struct SplitSmem {
    static constexpr int CH = chains(NP);
    static constexpr int NWALK = (CH + 31) / 32;
    static constexpr int WL = CH < 32 ? CH : 32;             // chains per walker warp
    static constexpr int NCUT_W = ISSUER_WARP - NWALK;        // cutter warps
    static constexpr int GEN = 0;                             // 2 stages x DIG x A_TILE
    static constexpr int MAP_ST = 3;                          // map digit stages
    static constexpr int MAP = GEN + 2 * DIG * A_TILE;        // MAP_ST stages x DIG x B_TILE
    static constexpr int VB = MAP + MAP_ST * DIG * B_TILE;    // 2 x [64 chains][33]
    static constexpr int VB_ONE = 64 * 33;                    // doubles per buffer
    // walker tables, per walker warp and buffer (doubles): Ap[KC][WL], Am[KC], Om[KC]
    static constexpr int WT = VB + 2 * VB_ONE * 8;
    static constexpr int WT_AP = 0, WT_AM = KC * WL, WT_OM = WT_AM + KC, WT_DBL = WT_OM + KC;
    // factor tables of the cutters, per buffer (doubles): G[KC][NP][CH]
    static constexpr int GT = WT + NWALK * 2 * WT_DBL * 8;
    static constexpr int GT_DBL = KC * NP * CH;
    static constexpr int PH = GT + 2 * GT_DBL * 8;            // phases [g*16 + n+N-1]
    static constexpr int EF = PH + 8 * 16 * 16;               // column factors 2^(Ef - SHIFT)
    static constexpr int BAR = EF + COLS * 8;                 // VFULL[2], CUT[2], full[3], done[2]
    static constexpr int TM = BAR + 9 * 8;
    static constexpr int ABORT = TM + 8;
    static constexpr int BYTES = ABORT + 8 + 1024;            // + alignment slack
    static constexpr int TS_LD = COLS + 1;                    // epilogue tile row stride
    static_assert(ROWS * TS_LD * 8 <= WT, "epilogue tile fits the operand and value buffers");
    static_assert(LEV * COLS <= TMEM_COLS, "level accumulators fit TMEM");
    static_assert(NCUT_W * 32 >= 128, "one cutting item per cutter thread");
};

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void named_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }

template <int NP>
__global__ void __launch_bounds__(SPLIT_THREADS, 1) split_kernel(SplitArgs a)
{
    using S = SplitSmem<NP>;
    constexpr int CH = S::CH, NWALK = S::NWALK, WL = S::WL;
    constexpr int PAIRS = CH * NP;  // <= 64
    constexpr int NCT = S::NCUT_W * 32;
    extern __shared__ unsigned char smraw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
    double2 *sPh = reinterpret_cast<double2 *>(sm + S::PH);
    double *sFc = reinterpret_cast<double *>(sm + S::EF);
    uint32_t *sTm = reinterpret_cast<uint32_t *>(sm + S::TM);
    volatile int *sAbort = reinterpret_cast<volatile int *>(sm + S::ABORT);
    const uint32_t bar0 = smem_u32(sm + S::BAR);
    auto vfull = [&](int b) { return bar0 + 8 * b; };
    auto cutb = [&](int b) { return bar0 + 16 + 8 * b; };
    auto full = [&](int b) { return bar0 + 32 + 8 * b; };
    auto done = [&](int b) { return bar0 + 56 + 8 * b; };
    // bounded wait that returns at once after an abort
    auto wait = [&](uint32_t bar, uint32_t parity) -> bool {
        if (*sAbort) return false;
        if (mbar_try(bar, parity)) return true;
        const unsigned long long t0 = gtimer();
        while (true) {
            if (mbar_try(bar, parity)) return true;
            if (*sAbort || gtimer() - t0 > a.wait_ns) {
                *sAbort = 1;
                return false;
            }
        }
    };

    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int2 tile = a.tiles[blockIdx.x];
    const int m = tile.x, p0 = tile.y * CH;
    const int bl = a.bl, blo = a.blo, N = a.N;
    const int lw = max(m, p0);        // first row any chain walks
    const int lk = max(blo + 1, lw);  // first row with output
    const int cw0 = lw / KC, c_last = (bl - 1) / KC;
    const int c_start = lk / KC;
    const bool has_mma = lk < bl;
    const int nout = has_mma ? c_last - c_start + 1 : 0;

    // ---- setup
    if (t == 0) {
        for (int i = 0; i < 2; i++) {
            mbar_init(vfull(i), NWALK);
            mbar_init(cutb(i), S::NCUT_W);
            mbar_init(done(i), 1);
        }
        for (int i = 0; i < S::MAP_ST; i++) mbar_init(full(i), 1);
        mbar_fence_init();
        *sAbort = 0;
    }
    if (warp == 0) {
        tmem_alloc(smem_u32(sTm), TMEM_COLS);
        tmem_relinquish();
    }
    for (int i = t; i < N * 16; i += SPLIT_THREADS) sPh[i] = a.ph[i];
    if (t < COLS) {
        const int Ef = a.fexp[(size_t)m * COLS + t];
        sFc[t] = Ef > E_MIN ? pow2i(Ef - SHIFT) : 0.0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *sTm;

    if (warp < NWALK) {
        // ================= walker =================
        const int ch = warp * 32 + lane;  // chain of this lane
        const bool walker = lane < WL && ch < CH;
        const int wmp = p0 + ch;
        Chain cn = chain_init(a.Ste, a.Stm, a.B, m, wmp, walker && wmp < bl);
        double *WT = reinterpret_cast<double *>(sm + S::WT) + warp * 2 * S::WT_DBL;
        // staging: a fixed pattern per lane (its 16-byte piece of an Ap row,
        // rows in passes; one row of Am and Om), so that a copy costs a row
        // bound check and one address computation
        static_assert(KC == 32 && (WL == 16 || WL == 32), "walker staging pattern");
        constexpr int V = WL / 2, RP = 32 / V;  // pieces per Ap row, rows per pass
        const int pc = lane % V, col = p0 + warp * 32 + 2 * pc;
        const bool colok = col < a.Bp;
        auto stage = [&](int c, int b) {
            double *T = WT + b * S::WT_DBL;
            const int lb = c * KC;
#pragma unroll
            for (int k = 0; k < KC / RP; k++) {
                const int li = lane / V + RP * k, l = lb + li;
                double *d = T + S::WT_AP + li * WL + 2 * pc;
                if (l < bl && colok) cp_async16(d, a.Acoef + (size_t)l * a.Bp + col);
                else { d[0] = 0.0; d[1] = 0.0; }
            }
            const int l = lb + lane;
            double *dm = T + S::WT_AM + lane, *dom = T + S::WT_OM + lane;
            if (l < bl) {
                cp_async8(dm, a.Acoef + (size_t)l * a.Bp + m);
                cp_async8(dom, a.Om + (size_t)l * a.Bp + m);
            } else {
                *dm = 0.0;
                *dom = 0.0;
            }
        };
        if (has_mma) {
            stage(cw0, 0);
            cp_commit_all();
            for (int c = cw0; c <= c_last; c++) {
                const int wb = (c - cw0) & 1;
                if (c + 1 <= c_last) stage(c + 1, wb ^ 1);
                cp_commit_all();
                asm volatile("cp.async.wait_group 1;" ::: "memory");
                __syncwarp();
                const double *T = WT + wb * S::WT_DBL;
                const int k = c - c_start;
                const bool out = k >= 0;
                if (out && k >= 2) wait(cutb(k & 1), ((k - 2) >> 1) & 1);  // cutters done with chunk k-2
                const int lb = c * KC;
                const int lo = max(lb, lw) - lb, hi = min(lb + KC, bl) - lb;
                double *vrow = reinterpret_cast<double *>(sm + S::VB) + (k & 1) * S::VB_ONE + ch * 33;
                if (lo == 0 && hi == KC) {
                    double wv[KC];
#pragma unroll
                    for (int li = 0; li < KC; li++) {
                        wv[li] = chain_step(cn, lb + li, T[S::WT_AM + li], walker ? T[S::WT_AP + li * WL + lane] : 0.0,
                                            T[S::WT_OM + li]);
                        if ((li & 15) == 15) chain_renorm(cn);
                    }
                    if (out && walker) {
#pragma unroll
                        for (int li = 0; li < KC; li++) vrow[li] = wv[li];
                    }
                } else {
                    for (int li = 0; li < KC; li++) {
                        const int l = lb + li;
                        double w = 0.0;
                        if (li >= lo && li < hi) {
                            w = chain_step(cn, l, T[S::WT_AM + li], walker ? T[S::WT_AP + li * WL + lane] : 0.0,
                                           T[S::WT_OM + li]);
                            if ((l & 15) == 15) chain_renorm(cn);
                        }
                        if (out && walker) vrow[li] = w;
                    }
                }
                __syncwarp();
                if (out && lane == 0) mbar_arrive(vfull(k & 1));
            }
            cp_wait_all();
        }
    } else if (warp < ISSUER_WARP) {
        // ================= cutters =================
        const int ct = t - NWALK * 32;
        const bool item = ct < 128;
        const int pair = ct >> 1, kh = ct & 1;
        const int pch = pair / NP, pq = pair % NP, pmp = p0 + pch;
        const bool prow = item && pair < PAIRS && pmp < bl;
        const int Ed = prow ? (int)a.dexp[((size_t)m * bl + pmp) * NP + pq] : E_ZERO;
        const double dfac = digit_factor(Ed);
        double *GT = reinterpret_cast<double *>(sm + S::GT);
        // staging: the cutter threads are a whole number of G row groups
        // (NP rows of CH doubles per l), so each thread copies a fixed piece
        // (q, x) of every RS-th l
        constexpr int V = CH / 2, RW = NP * V, RS = NCT / RW;
        static_assert(NCT % RW == 0, "cutter staging pattern");
        const int sq = (ct % RW) / V, sx = 2 * ((ct % RW) % V), li0 = ct / RW;
        const bool sxok = p0 + sx < a.Gs;
        auto stage = [&](int c, int b) {
            double *T = GT + b * S::GT_DBL;
            const int lb = c * KC;
            for (int li = li0; li < KC; li += RS) {
                const int l = lb + li;
                double *d = T + (li * NP + sq) * CH + sx;
                if (l < bl && l > blo && sxok)
                    cp_async16(d, a.G + ((size_t)(l - blo - 1) * NP + sq) * a.Gs + p0 + sx);
                else { d[0] = 0.0; d[1] = 0.0; }
            }
        };
        if (nout > 0) {
            stage(c_start, 0);
            cp_commit_all();
        }
        for (int k = 0; k < nout; k++) {
            const int c = c_start + k, gb = k & 1;
            if (k + 1 < nout) stage(c + 1, gb ^ 1);
            cp_commit_all();
            asm volatile("cp.async.wait_group 1;" ::: "memory");
            named_sync(1, NCT);  // G of chunk k visible to every cutter
            bool ok = wait(vfull(k & 1), (k >> 1) & 1);
            if (k >= 2) ok = wait(done(k & 1), ((k - 2) >> 1) & 1) && ok;  // MMAs of chunk k-2 finished
            if (ok && item) {
                const double *T = GT + gb * S::GT_DBL;
                const double *vb = reinterpret_cast<const double *>(sm + S::VB) + (k & 1) * S::VB_ONE;
                unsigned char *gen = sm + S::GEN + (k & 1) * DIG * A_TILE;
                const int lb = c * KC;
                long long X[16];
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const int li = 16 * kh + i, l = lb + li;
                    double v = 0.0;
                    if (prow && l > blo) v = vb[pch * 33 + li] * T[(li * NP + pq) * CH + pch];
                    X[i] = to_fixed(v, dfac);
                }
                // rows 2 pair (even l) and 2 pair + 1 (odd l): the epilogue
                // forms E + O and E - O, the +n and -n sums; l = 32c + 16kh + i
                store_digits_parity(gen + tile_off(ROWS, 2 * pair, kh), gen + tile_off(ROWS, 2 * pair + 1, kh),
                                    A_TILE, X);
                fence_async_smem();
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(cutb(k & 1));
            named_sync(1, NCT);  // every cutter finished with G buffer gb
        }
        cp_wait_all();
    } else if (lane == 0 && nout > 0) {
        // ================= issuer =================
        // copies issued into / consumed from each map stage, last MMA commit:
        // what the drain after an abort must wait for
        int ncopy[S::MAP_ST] = {}, nused[S::MAP_ST] = {}, last_commit = -1;
        auto map_copy = [&](int c) {
            const int st = (c - c_start) % S::MAP_ST;
            mbar_expect_tx(full(st), DIG * B_TILE);
            bulk_g2s(smem_u32(sm + S::MAP + st * DIG * B_TILE),
                     a.fdig + ((size_t)m * a.nch + (c - a.c0)) * DIG * B_TILE, DIG * B_TILE, full(st));
            ncopy[st]++;
        };
        const uint32_t idesc_uu = idesc_i8(0, 0, ROWS, COLS), idesc_su = idesc_i8(1, 0, ROWS, COLS),
                       idesc_us = idesc_i8(0, 1, ROWS, COLS), idesc_ss = idesc_i8(1, 1, ROWS, COLS);
        bool first_lev[LEV];
#pragma unroll
        for (int i = 0; i < LEV; i++) first_lev[i] = true;
        // Map digits run two chunks ahead in three stages: the copy for chunk
        // k + 2 goes into the stage the MMAs of chunk k - 1 read, once those
        // have finished, so that the MMAs of chunk k are issued without
        // waiting for chunk k - 1's to complete.
        map_copy(c_start);
        if (nout > 1) map_copy(c_start + 1);
        for (int k = 0; k < nout; k++) {
            const int gs = k & 1, ms = k % S::MAP_ST, c = c_start + k;
            if (!wait(cutb(gs), (k >> 1) & 1)) continue;
            if (!wait(full(ms), (k / S::MAP_ST) & 1)) continue;
            nused[ms]++;
            tc_fence_after();
            const uint64_t da0 = smem_desc(smem_u32(sm + S::GEN + gs * DIG * A_TILE), ROWS * 16, 128);
            const uint64_t db0 = smem_desc(smem_u32(sm + S::MAP + ms * DIG * B_TILE), COLS * 16, 128);
#pragma unroll
            for (int i = 0; i < DIG; i++)
#pragma unroll
                for (int j = 0; j < DIG; j++) {
                    const int lev = 2 * (DIG - 1) - i - j;
                    if (lev >= LEV) continue;
                    const uint32_t id = (i == DIG - 1) ? (j == DIG - 1 ? idesc_ss : idesc_su)
                                                       : (j == DIG - 1 ? idesc_us : idesc_uu);
                    mma_i8(tmem + lev * COLS, da0 + (uint64_t)((i * A_TILE) >> 4),
                           db0 + (uint64_t)((j * B_TILE) >> 4), id, first_lev[lev] ? 0u : 1u);
                    first_lev[lev] = false;
                }
            mma_commit(done(gs));
            last_commit = k;
            if (k + 2 < nout) {
                if (k >= 1 && !wait(done(gs ^ 1), ((k - 1) >> 1) & 1)) continue;
                map_copy(c + 2);
            }
        }
        if (!wait(done((nout - 1) & 1), ((nout - 1) >> 1) & 1)) {
            // a wait gave up: let this CTA's copies and MMAs in flight finish
            // before its shared memory and TMEM are released.  At most one
            // copy per stage is unconsumed; the commit of chunk k is phase
            // k/2 of done(k%2).
            for (int st = 0; st < S::MAP_ST; st++)
                if (ncopy[st] > nused[st]) drain_wait(full(st), (ncopy[st] - 1) & 1);
            if (last_commit >= 0) drain_wait(done(last_commit & 1), (last_commit >> 1) & 1);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    const bool abort = *sAbort != 0;
    if (abort && t == 0) atomicExch(a.err, 1);

    // ---- epilogue: warp w reads TMEM lanes 32*(w&3).. (rows) and columns
    // [32*(w>>2), +32) (maps 16*(w>>2) .. +16)
    double *Ts = reinterpret_cast<double *>(sm + S::GEN);  // [row * TS_LD + col]
    {
        const int row = 32 * (warp & 3) + lane, half = warp >> 2;
        const int rp = row >> 1, rch = rp / NP, rq = rp % NP, rmp = p0 + rch;
        const int Er = (rp < PAIRS && rmp < bl) ? (int)a.dexp[((size_t)m * bl + rmp) * NP + rq] : E_ZERO;
        const double rowf = Er > E_MIN ? pow2i(Er) : 0.0;
        for (int blk = 0; blk < 2; blk++) {
            const int col0 = 32 * half + 16 * blk;
            double acc[16];
#pragma unroll
            for (int i = 0; i < 16; i++) acc[i] = 0.0;
            if (nout > 0 && !abort) {
                int32_t r[LEV][16];
                tmem_ld16x7(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + col0, r);
#pragma unroll
                for (int lev = 0; lev < LEV; lev++) {
                    const double wgt = pow2i(-8 * lev);
#pragma unroll
                    for (int i = 0; i < 16; i++) acc[i] = fma((double)r[lev][i], wgt, acc[i]);
                }
            }
#pragma unroll
            for (int i = 0; i < 16; i++) Ts[row * S::TS_LD + col0 + i] = (acc[i] * rowf) * sFc[col0 + i];
        }
    }
    __syncthreads();
    // (chain, map) items
    const int ev = (N % 2 == 0) ? 1 : 0;
    constexpr int ITEMS = CH * MAPS;
    for (int it = t; it < ITEMS; it += SPLIT_THREADS) {
        const int c = it % CH, k = it / CH, mp = p0 + c;
        if (mp >= bl || k >= a.nmaps) continue;
        double2 Tp[NP], Tm[NP];
#pragma unroll
        for (int q = 0; q < NP; q++) {
            const int n = a.nq[q], pr = c * NP + q;
            // rows 2 pr and 2 pr + 1 hold the even-l and odd-l sums E, O
            const double2 E = make_double2(Ts[(2 * pr) * S::TS_LD + 2 * k], Ts[(2 * pr) * S::TS_LD + 2 * k + 1]);
            const double2 O =
                make_double2(Ts[(2 * pr + 1) * S::TS_LD + 2 * k], Ts[(2 * pr + 1) * S::TS_LD + 2 * k + 1]);
            const double2 sum = make_double2(E.x + O.x, E.y + O.y), dif = make_double2(E.x - O.x, E.y - O.y);
            if (n == 0) {
                Tp[q] = c_ipow(sum, -m);
                Tm[q] = make_double2(0.0, 0.0);
            } else {
                Tp[q] = c_ipow(sum, n - m - ev);
                double2 x = c_ipow(dif, -n - m + ev);
                if ((mp + n) & 1) x = make_double2(-x.x, -x.y);
                Tm[q] = x;
            }
        }
        double2 *out = a.Tg + (size_t)k * N * bl * bl;
        for (int g = 0; g < N; g++) {
            double2 y = make_double2(0.0, 0.0);
#pragma unroll
            for (int q = 0; q < NP; q++) {
                const int n = a.nq[q];
                y = c_add(y, c_mul(Tp[q], sPh[g * 16 + n + N - 1]));
                if (n != 0) y = c_add(y, c_mul(Tm[q], sPh[g * 16 - n + N - 1]));
            }
            out[((size_t)g * bl + m) * bl + mp] = y;
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, TMEM_COLS);
}

// ===========================================================================
// Synthesis: the contraction of s2dw_core_mod.f90:1200-1253 for a batch,
//
//   part^k(l, m) = i^m sum_{m' <= l} sum_q v(m'; l, m, q) V^k(q, m, m'),
//   v = d^l_{m'm}(pi/2) d^l_{m'n_q}(pi/2) c_j(l, n_q),
//
// a GEMM per m with rows l (chains of the m'-recurrence, 128 per CTA), K over
// (m', q) and columns (map, re/im).  Same digits, levels and TMEM layout as
// the analysis; the walker warps cut their own rows (no parity rows here).
// ===========================================================================
__host__ __device__ constexpr int syn_npq(int NP) { return NP == 1 ? 1 : (NP == 2 ? 2 : 4); }
__host__ __device__ constexpr int syn_mc(int NP) { return KC / syn_npq(NP); }
constexpr int SYN_ROWS = 128;

// m'-walk of chain (l, m): the recurrence of mwalk_kernel, e_{m'-1} =
// m b(l,m') e_{m'} - e_{m'+1}, started at m' = l.
__device__ __forceinline__ Chain syn_chain_init(const int32_t *Ee, const double *Em, int B, int l, int m, bool valid)
{
    Chain c;
    c.e = 0.0;
    c.ep = 0.0;
    c.st = 0.0;
    c.l0 = valid ? l : INT_MAX;
    int maxe = valid ? (int)Ee[(size_t)l * B + m] : INT_MIN;
    maxe = wmax_i(maxe);
    c.Kw = (maxe != INT_MIN && maxe < S2DW_SCALE_EXP) ? -maxe : 0;
    c.sc = pow2_or_zero(-c.Kw);
    if (valid) {
        const double v = ldexp(Em[(size_t)l * B + m], (int)Ee[(size_t)l * B + m] + c.Kw);
        c.st = ((l - m) & 1) ? -v : v;
    }
    return c;
}
// value at m' (true scale), then one step down; p = m b(l, m')
__device__ __forceinline__ double syn_chain_step(Chain &c, int mp, double p)
{
    if (mp == c.l0) c.e = c.st;
    const double w = c.e * c.sc;
    const double en = fma(p, c.e, -c.ep);
    c.ep = c.e;
    c.e = en;
    return w;
}

// sexp: exponent of max over (m', q) of |v| per chain; one CTA per tile.
template <int NP>
__global__ void __launch_bounds__(SYN_ROWS) syn_dexp_kernel(SplitSynArgs a)
{
    const int2 tile = a.tiles[blockIdx.x];
    const int m = tile.x, lbase = a.blo + 1 + tile.y * SYN_ROWS;
    const int l = lbase + threadIdx.x;
    const int MH = min(lbase + SYN_ROWS - 1, a.bl - 1);
    const bool valid = l < a.bl && m <= l;
    Chain c = syn_chain_init(a.Ee, a.Em, a.B, l, m, valid);
    const int lc = min(l, a.bl - 1);
    const double mm = (double)m;
    double mx = 0.0;
#pragma unroll 4
    for (int mp = MH; mp >= 0; mp--) {
        const double w = syn_chain_step(c, mp, mm * a.Bcoef[(size_t)lc * a.Bp + mp]);
        if (valid && mp <= l) {
#pragma unroll
            for (int q = 0; q < NP; q++)
                mx = fmax(mx, fabs(w * a.G[((size_t)(l - a.blo - 1) * NP + q) * a.Gs + mp]));
        }
        if ((mp & 15) == 0) chain_renorm(c);
    }
    if (valid) a.sexp[(size_t)m * a.bl + l] = (int16_t)(mx > 0.0 ? ilogb(mx) + 1 : E_ZERO);
}

// Map digits of the synthesis: column col = 2k + (re, im) of V^k(q, m, m');
// K index within chunk ci: kk = (m' - MC ci) * NPQ + q.  One CTA per m.
template <int NP>
__global__ void __launch_bounds__(THREADS) vdig_kernel(VdigArgs a)
{
    constexpr int NPQ = syn_npq(NP), MC = syn_mc(NP);
    __shared__ int sE[COLS];
    const int m = blockIdx.x, t = threadIdx.x;
    const int col = t >> 1, half = t & 1, k = col >> 1, comp = col & 1;
    const double *V = reinterpret_cast<const double *>(a.V2f + (size_t)k * a.vstride) + comp;
    double mx = 0.0;
    if (k < a.nmaps)
        for (int q = 0; q < NP; q++)
            for (int mp = half; mp < a.bl; mp += 2)
                mx = fmax(mx, fabs(V[2 * (((size_t)q * a.bl + m) * a.Vs + mp)]));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
    const int E = mx > 0.0 ? ilogb(mx) + 1 : E_ZERO;
    if (half == 0) {
        sE[col] = E;
        a.vexp[(size_t)m * COLS + col] = E;
    }
    __syncthreads();
    const double factor = digit_factor(sE[col]);
    const int kh = half;
    for (int ci = 0; ci < a.nch; ci++) {
        long long X[16];
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const int kk = 16 * kh + i, q = kk % NPQ, mp = ci * MC + kk / NPQ;
            const double v = (k < a.nmaps && q < NP && mp < a.bl) ? V[2 * (((size_t)q * a.bl + m) * a.Vs + mp)] : 0.0;
            X[i] = to_fixed(v, factor);
        }
        unsigned char *dst = a.vdig + ((size_t)m * a.nch + ci) * DIG * B_TILE + tile_off(COLS, col, kh);
        store_digits(dst, B_TILE, X);
    }
}

template <int NP>
struct SynSmem {
    static constexpr int NPQ = syn_npq(NP), MC = syn_mc(NP);
    static constexpr int RS = MC + 2;                         // padded table row (16-byte aligned)
    static constexpr int GEN = 0;                             // 2 stages x DIG x A_TILE
    static constexpr int MAP = GEN + 2 * DIG * A_TILE;        // 2 stages x DIG x B_TILE
    // lane-private staged rows per buffer (doubles): b[128][RS], G[128][NP][RS]
    static constexpr int TB = MAP + 2 * DIG * B_TILE;
    static constexpr int T_B = 0, T_G = SYN_ROWS * RS, T_DBL = T_G + SYN_ROWS * NP * RS;
    static constexpr int EF = TB + 2 * T_DBL * 8;
    static constexpr int BAR = EF + COLS * 8;                 // gfull[2], full[2], done[2]
    static constexpr int TM = BAR + 6 * 8;
    static constexpr int ABORT = TM + 8;
    static constexpr int BYTES = ABORT + 8 + 1024;
    static_assert(LEV * COLS <= TMEM_COLS, "level accumulators fit TMEM");
    static_assert(BYTES <= 227 * 1024, "shared memory");
};

// Roles (256 threads): warps 0-3 walk the 128 chains and cut their own rows;
// warp 7 lane 0 issues the map copies and MMAs; all warps run the epilogue.
template <int NP>
__global__ void __launch_bounds__(SPLIT_THREADS, 1) split_syn_kernel(SplitSynArgs a)
{
    using S = SynSmem<NP>;
    constexpr int NPQ = S::NPQ, MC = S::MC, RS = S::RS;
    extern __shared__ unsigned char smraw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
    double *sFc = reinterpret_cast<double *>(sm + S::EF);
    uint32_t *sTm = reinterpret_cast<uint32_t *>(sm + S::TM);
    volatile int *sAbort = reinterpret_cast<volatile int *>(sm + S::ABORT);
    const uint32_t bar0 = smem_u32(sm + S::BAR);
    auto gfull = [&](int b) { return bar0 + 8 * b; };
    auto full = [&](int b) { return bar0 + 16 + 8 * b; };
    auto done = [&](int b) { return bar0 + 32 + 8 * b; };
    auto wait = [&](uint32_t bar, uint32_t parity) -> bool {
        if (*sAbort) return false;
        if (mbar_try(bar, parity)) return true;
        const unsigned long long t0 = gtimer();
        while (true) {
            if (mbar_try(bar, parity)) return true;
            if (*sAbort || gtimer() - t0 > a.wait_ns) {
                *sAbort = 1;
                return false;
            }
        }
    };

    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int2 tile = a.tiles[blockIdx.x];
    const int m = tile.x, lbase = a.blo + 1 + tile.y * SYN_ROWS;
    const int bl = a.bl;
    const int MH = min(lbase + SYN_ROWS - 1, bl - 1);
    const int ctop = MH / MC;
    const int nck = ctop + 1;  // chunks ctop, ctop-1, ..., 0

    if (t == 0) {
        for (int i = 0; i < 2; i++) {
            mbar_init(gfull(i), 4);
            mbar_init(full(i), 1);
            mbar_init(done(i), 1);
        }
        mbar_fence_init();
        *sAbort = 0;
    }
    if (warp == 0) {
        tmem_alloc(smem_u32(sTm), TMEM_COLS);
        tmem_relinquish();
    }
    if (t < COLS) {
        const int Ef = a.vexp[(size_t)m * COLS + t];
        sFc[t] = Ef > E_MIN ? pow2i(Ef - SHIFT) : 0.0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *sTm;

    if (warp < 4) {
        // ================= walkers / cutters =================
        const int l = lbase + t;
        const bool valid = l < bl && m <= l;
        Chain cn = syn_chain_init(a.Ee, a.Em, a.B, l, m, valid);
        const int Er = valid ? (int)a.sexp[(size_t)m * bl + l] : E_ZERO;
        const double dfac = digit_factor(Er);
        const double mm = (double)m;
        double *TBp = reinterpret_cast<double *>(sm + S::TB);
        // this lane's table rows of chunk c -> buffer b (lane-private)
        auto stage = [&](int c, int b) {
            double *T = TBp + b * S::T_DBL;
            const int m0 = c * MC;
            double *db = T + S::T_B + t * RS;
            for (int x = 0; x < MC; x += 2) {
                if (l < bl && m0 + x < a.Bp) cp_async16(db + x, a.Bcoef + (size_t)l * a.Bp + m0 + x);
                else { db[x] = 0.0; db[x + 1] = 0.0; }
            }
            for (int q = 0; q < NP; q++) {
                double *dg = T + S::T_G + (t * NP + q) * RS;
                for (int x = 0; x < MC; x += 2) {
                    if (valid && m0 + x < a.Gs)
                        cp_async16(dg + x, a.G + ((size_t)(l - a.blo - 1) * NP + q) * a.Gs + m0 + x);
                    else { dg[x] = 0.0; dg[x + 1] = 0.0; }
                }
            }
        };
        stage(ctop, 0);
        cp_commit_all();
        for (int k = 0; k < nck; k++) {
            const int c = ctop - k, tb = k & 1;
            if (k + 1 < nck) stage(c - 1, tb ^ 1);
            cp_commit_all();
            asm volatile("cp.async.wait_group 1;" ::: "memory");
            const double *T = TBp + tb * S::T_DBL;
            // walk m' = MC c + MC - 1 .. MC c (down), values v(m', q)
            double vals[KC];
#pragma unroll
            for (int i = 0; i < KC; i++) vals[i] = 0.0;
#pragma unroll
            for (int u = MC - 1; u >= 0; u -= 2) {
                const double2 bb = *reinterpret_cast<const double2 *>(T + S::T_B + t * RS + u - 1);
                double2 gg[NP];
#pragma unroll
                for (int q = 0; q < NP; q++)
                    gg[q] = *reinterpret_cast<const double2 *>(T + S::T_G + (t * NP + q) * RS + u - 1);
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int uu = u - h, mp = c * MC + uu;
                    if (mp <= MH) {
                        const double w = syn_chain_step(cn, mp, mm * (h == 0 ? bb.y : bb.x));
#pragma unroll
                        for (int q = 0; q < NP; q++) vals[uu * NPQ + q] = w * (h == 0 ? gg[q].y : gg[q].x);
                        if ((mp & 15) == 0) chain_renorm(cn);
                    }
                }
            }
            if (k >= 2) wait(done(k & 1), ((k - 2) >> 1) & 1);  // MMAs of chunk k-2 finished
            if (!*sAbort) {
                unsigned char *gen = sm + S::GEN + (k & 1) * DIG * A_TILE;
#pragma unroll
                for (int kh = 0; kh < 2; kh++) {
                    long long X[16];
#pragma unroll
                    for (int i = 0; i < 16; i++) X[i] = to_fixed(vals[16 * kh + i], dfac);
                    store_digits(gen + tile_off(ROWS, t, kh), A_TILE, X);
                }
                fence_async_smem();
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(gfull(k & 1));
        }
        cp_wait_all();
    } else if (warp == ISSUER_WARP && lane == 0) {
        // ================= issuer =================
        int ncopy[2] = {}, nused[2] = {}, last_commit = -1;  // for the drain after an abort
        auto map_copy = [&](int c, int st) {
            mbar_expect_tx(full(st), DIG * B_TILE);
            bulk_g2s(smem_u32(sm + S::MAP + st * DIG * B_TILE), a.vdig + ((size_t)m * a.nch + c) * DIG * B_TILE,
                     DIG * B_TILE, full(st));
            ncopy[st]++;
        };
        const uint32_t idesc_uu = idesc_i8(0, 0, ROWS, COLS), idesc_su = idesc_i8(1, 0, ROWS, COLS),
                       idesc_us = idesc_i8(0, 1, ROWS, COLS), idesc_ss = idesc_i8(1, 1, ROWS, COLS);
        bool first_lev[LEV];
#pragma unroll
        for (int i = 0; i < LEV; i++) first_lev[i] = true;
        map_copy(ctop, 0);
        for (int k = 0; k < nck; k++) {
            const int gs = k & 1, c = ctop - k;
            if (!wait(gfull(gs), (k >> 1) & 1)) continue;
            if (k >= 1 && !wait(done(gs ^ 1), ((k - 1) >> 1) & 1)) continue;
            if (k + 1 < nck) map_copy(c - 1, gs ^ 1);
            if (!wait(full(gs), (k >> 1) & 1)) continue;
            nused[gs]++;
            tc_fence_after();
            const uint64_t da0 = smem_desc(smem_u32(sm + S::GEN + gs * DIG * A_TILE), ROWS * 16, 128);
            const uint64_t db0 = smem_desc(smem_u32(sm + S::MAP + gs * DIG * B_TILE), COLS * 16, 128);
#pragma unroll
            for (int i = 0; i < DIG; i++)
#pragma unroll
                for (int j = 0; j < DIG; j++) {
                    const int lev = 2 * (DIG - 1) - i - j;
                    if (lev >= LEV) continue;
                    const uint32_t id = (i == DIG - 1) ? (j == DIG - 1 ? idesc_ss : idesc_su)
                                                       : (j == DIG - 1 ? idesc_us : idesc_uu);
                    mma_i8(tmem + lev * COLS, da0 + (uint64_t)((i * A_TILE) >> 4),
                           db0 + (uint64_t)((j * B_TILE) >> 4), id, first_lev[lev] ? 0u : 1u);
                    first_lev[lev] = false;
                }
            mma_commit(done(gs));
            last_commit = k;
        }
        if (!wait(done((nck - 1) & 1), ((nck - 1) >> 1) & 1)) {
            // as split_kernel: drain this CTA's copies and MMAs in flight
            for (int st = 0; st < 2; st++)
                if (ncopy[st] > nused[st]) drain_wait(full(st), (ncopy[st] - 1) & 1);
            if (last_commit >= 0) drain_wait(done(last_commit & 1), (last_commit >> 1) & 1);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    const bool abort = *sAbort != 0;
    if (abort && t == 0) atomicExch(a.err, 1);

    // ---- epilogue: warp w reads rows 32*(w&3).. and columns [32*(w>>2), +32)
    {
        const int row = 32 * (warp & 3) + lane, half = warp >> 2;
        const int l = lbase + row;
        const bool valid = l < bl && m <= l;
        const int Er = valid ? (int)a.sexp[(size_t)m * bl + l] : E_ZERO;
        const double rowf = Er > E_MIN ? pow2i(Er) : 0.0;
        for (int blk = 0; blk < 2; blk++) {
            const int col0 = 32 * half + 16 * blk;
            double acc[16];
#pragma unroll
            for (int i = 0; i < 16; i++) acc[i] = 0.0;
            if (!abort) {
                int32_t r[LEV][16];
                tmem_ld16x7(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + col0, r);
#pragma unroll
                for (int lev = 0; lev < LEV; lev++) {
                    const double wgt = pow2i(-8 * lev);
#pragma unroll
                    for (int i = 0; i < 16; i++) acc[i] = fma((double)r[lev][i], wgt, acc[i]);
                }
            }
            if (valid) {
#pragma unroll
                for (int i = 0; i < 16; i += 2) {
                    const int k = (col0 + i) >> 1;
                    if (k < a.nmaps) {
                        const double2 z = make_double2((acc[i] * rowf) * sFc[col0 + i], (acc[i + 1] * rowf) * sFc[col0 + i + 1]);
                        a.part[(size_t)k * a.pstride + (size_t)(l - a.blo - 1) * bl + m] = c_ipow(z, m);
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, TMEM_COLS);
}

}  // namespace split

int split_chains(int NP) { return split::chains(NP); }
int split_maps_per_pass() { return split::MAPS; }
long long split_fdig_bytes(int bl, int nch) { return (long long)bl * nch * split::DIG * split::B_TILE; }

int launch_split_dexp(const SplitArgs &a, cudaStream_t s)
{
    if (a.ntiles <= 0) return S2DWC_OK;
    const int thr = split::chains(a.NP) > 32 ? 64 : 32;
    switch (a.NP) {
    case 1: split::dexp_kernel<1><<<a.ntiles, thr, 0, s>>>(a); break;
    case 2: split::dexp_kernel<2><<<a.ntiles, thr, 0, s>>>(a); break;
    case 3: split::dexp_kernel<3><<<a.ntiles, thr, 0, s>>>(a); break;
    default: split::dexp_kernel<4><<<a.ntiles, thr, 0, s>>>(a); break;
    }
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

int launch_split_fdig(const FdigArgs &a, cudaStream_t s)
{
    if (a.bl <= 0 || a.nch <= 0) return S2DWC_OK;
    split::fdig_kernel<<<a.bl, split::THREADS, 0, s>>>(a);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

template <int NP>
static int launch_split_t(const SplitArgs &a, cudaStream_t s)
{
    const int bytes = split::SplitSmem<NP>::BYTES;
    static bool attr = false;
    if (!attr) {
        S2DW_CUDA_TRY(cudaFuncSetAttribute(split::split_kernel<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        attr = true;
    }
    split::split_kernel<NP><<<a.ntiles, split::SPLIT_THREADS, bytes, s>>>(a);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

int launch_split(const SplitArgs &a, cudaStream_t s)
{
    if (a.ntiles <= 0) return S2DWC_OK;
    switch (a.NP) {
    case 1: return launch_split_t<1>(a, s);
    case 2: return launch_split_t<2>(a, s);
    case 3: return launch_split_t<3>(a, s);
    default: return launch_split_t<4>(a, s);
    }
}


int split_syn_mc(int NP) { return split::syn_mc(NP); }
long long split_vdig_bytes(int bl, int nch) { return (long long)bl * nch * split::DIG * split::B_TILE; }

int launch_split_syn_dexp(const SplitSynArgs &a, cudaStream_t s)
{
    if (a.ntiles <= 0) return S2DWC_OK;
    switch (a.NP) {
    case 1: split::syn_dexp_kernel<1><<<a.ntiles, split::SYN_ROWS, 0, s>>>(a); break;
    case 2: split::syn_dexp_kernel<2><<<a.ntiles, split::SYN_ROWS, 0, s>>>(a); break;
    case 3: split::syn_dexp_kernel<3><<<a.ntiles, split::SYN_ROWS, 0, s>>>(a); break;
    default: split::syn_dexp_kernel<4><<<a.ntiles, split::SYN_ROWS, 0, s>>>(a); break;
    }
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

int launch_split_vdig(const VdigArgs &a, cudaStream_t s)
{
    if (a.bl <= 0 || a.nch <= 0) return S2DWC_OK;
    switch (a.NP) {
    case 1: split::vdig_kernel<1><<<a.bl, split::THREADS, 0, s>>>(a); break;
    case 2: split::vdig_kernel<2><<<a.bl, split::THREADS, 0, s>>>(a); break;
    case 3: split::vdig_kernel<3><<<a.bl, split::THREADS, 0, s>>>(a); break;
    default: split::vdig_kernel<4><<<a.bl, split::THREADS, 0, s>>>(a); break;
    }
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

template <int NP>
static int launch_split_syn_t(const SplitSynArgs &a, cudaStream_t s)
{
    const int bytes = split::SynSmem<NP>::BYTES;
    static bool attr = false;
    if (!attr) {
        S2DW_CUDA_TRY(
            cudaFuncSetAttribute(split::split_syn_kernel<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        attr = true;
    }
    split::split_syn_kernel<NP><<<a.ntiles, split::SPLIT_THREADS, bytes, s>>>(a);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

int launch_split_syn(const SplitSynArgs &a, cudaStream_t s)
{
    if (a.ntiles <= 0) return S2DWC_OK;
    switch (a.NP) {
    case 1: return launch_split_syn_t<1>(a, s);
    case 2: return launch_split_syn_t<2>(a, s);
    case 3: return launch_split_syn_t<3>(a, s);
    default: return launch_split_syn_t<4>(a, s);
    }
}

}  // namespace s2dw
