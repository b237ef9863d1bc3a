// Device kernels of libs2dw_cuda (sm_100a, FP64).
//
//  * lwalk_kernel  : analysis l-contraction T(m,m',n) = sum_l d^l_{m'm} d^l_{m'n} f_lm psi_ln
//                    (s2dw_core_mod.f90:625-673), fused with the gamma DFT
//                    (:679-705).  d^l_{m'm}(pi/2) is generated in registers by
//                    a three-term recurrence in l, one plane per step, never
//                    stored.
//  * mwalk_kernel  : synthesis contraction wig(l,m,n) = sum_m' V d^l_{m'm} d^l_{m'n}
//                    and harmonic accumulation (:1200-1253), generating d by a
//                    recurrence in m' at fixed (l,m).
//  * czt_kernel    : chirp-z (Bluestein) transforms in shared memory that
//                    replace the naive beta sums (:708-743, :1157-1198) and
//                    the FFTW alpha transforms (:746-768, :1104-1130).
#include <cuda_runtime.h>

#include <climits>
#include <cstdio>
#include <type_traits>

#include "s2dw_internal.h"

namespace s2dw {

// ---------------------------------------------------------------------------
// Complex helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// z * i^k
__device__ __forceinline__ double2 cipow(double2 z, int k)
{
    switch (k & 3) {
    case 0: return z;
    case 1: return make_double2(-z.y, z.x);
    case 2: return make_double2(-z.x, -z.y);
    default: return make_double2(z.y, -z.x);
    }
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int warp_max_i(int v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Exponent below which a warp works in a scaled domain: start values below
// 2^-600 are multiplied by 2^Kw so that the recurrence cannot underflow
// (B > ~1000 has edge values down to 2^-B).
#define S2DW_SCALE_EXP (-600)
#define S2DW_RENORM_EXP 400

// ===========================================================================
// Asynchronous global -> shared copies (16 bytes, L2 only)
// ===========================================================================
__device__ __forceinline__ void cp16(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// ===========================================================================
// Analysis: l-walk contraction fused with the gamma DFT
//
// CTA tile: 32 consecutive m' (lanes) x LW_W*S consecutive m (S per warp).
// Each thread walks l for its S pairs (m', m); per step it needs a(l,m'),
// G(l,m',q) (lane-distinct) and a(l,m), F(l,m) (warp-uniform broadcast),
// staged LW_CH values of l at a time in a double-buffered cp.async pipeline.
// ===========================================================================
constexpr int LW_W = 4;    // warps per CTA
constexpr int LW_CH = 16;  // l values per staged chunk (even)

template <int NP, int S>
struct LwalkSmem {
    static constexpr int WS = LW_W * S;
    // per buffer, in doubles: F (complex, first for 16-byte alignment), Ap, G, Am
    static constexpr int F_OFF = 0;
    static constexpr int AP_OFF = F_OFF + 2 * LW_CH * WS;
    static constexpr int G_OFF = AP_OFF + LW_CH * 32;
    static constexpr int AM_OFF = G_OFF + LW_CH * NP * 32;
    static constexpr int BUF = AM_OFF + LW_CH * WS;
    static constexpr size_t BYTES = 2 * BUF * sizeof(double) + 8 * 16 * sizeof(double2);
};

template <int NP, int S>
__global__ void __launch_bounds__(LW_W * 32) lwalk_kernel(LwalkArgs a, int tiles_p)
{
    using L = LwalkSmem<NP, S>;
    constexpr int WS = L::WS;
    extern __shared__ __align__(16) double lsm[];
    double2 *sPh = reinterpret_cast<double2 *>(lsm + 2 * L::BUF);  // [g*16 + n+N-1]

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int pt = blockIdx.x % tiles_p, mt = blockIdx.x / tiles_p;
    const int p0 = pt * 32, m0 = mt * WS;
    const int B = a.B, Bp = a.Bp, bl = a.bl, blo = a.blo, N = a.N, Gs = a.Gs;
    const int mp = p0 + lane;

    for (int i = tid; i < N * (2 * N - 1); i += blockDim.x) {
        const int g = i / (2 * N - 1), n = i % (2 * N - 1) - (N - 1);
        double sn, cs;
        sincospi((double)(n * g) / (double)N, &sn, &cs);
        sPh[g * 16 + n + N - 1] = make_double2(cs, sn);
    }

    // ---- per-pair start values; pair = (m' = mp, m = m0 + w*S + s)
    int l0[S];
    double st[S];
    int maxe = INT_MIN;
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int m = m0 + w * S + s;
        const bool valid = (mp < bl) && (m < bl);
        l0[s] = valid ? max(mp, m) : INT_MAX;
        if (valid) maxe = max(maxe, (int)a.Ste[(size_t)max(mp, m) * B + min(mp, m)]);
    }
    maxe = warp_max_i(maxe);
    int Kw = (maxe != INT_MIN && maxe < S2DW_SCALE_EXP) ? -maxe : 0;
#pragma unroll
    for (int s = 0; s < S; s++) {
        const int m = m0 + w * S + s;
        st[s] = 0.0;
        if (l0[s] != INT_MAX) {
            const size_t o = (size_t)l0[s] * B + min(mp, m);
            double v = ldexp(a.Stm[o], (int)a.Ste[o] + Kw);
            if (mp >= m && ((mp - m) & 1)) v = -v;
            st[s] = v;
        }
    }

    double e[S], ep[S];
    double2 acc[2][S][NP];
#pragma unroll
    for (int s = 0; s < S; s++) {
        e[s] = 0.0;
        ep[s] = 0.0;
#pragma unroll
        for (int q = 0; q < NP; q++) acc[0][s][q] = acc[1][s][q] = make_double2(0.0, 0.0);
    }

    const int lstart = max(p0, m0) & ~1;
    const int rampEnd = min(max(p0 + 31, m0 + WS - 1), bl - 1);
    const int nchunks = (bl - lstart + LW_CH - 1) / LW_CH;

    auto stage = [&](int c, int buf) {
        const int lc = lstart + c * LW_CH;
        double *b = lsm + buf * L::BUF;
        // a(l, m') and a(l, m): 32 and WS doubles per row
        for (int i = tid; i < LW_CH * (16 + WS / 2); i += blockDim.x) {
            const int li = i / (16 + WS / 2), r = i % (16 + WS / 2), l = lc + li;
            if (l >= bl) continue;
            if (r < 16) cp16(b + L::AP_OFF + li * 32 + 2 * r, a.Acoef + (size_t)l * Bp + p0 + 2 * r);
            else cp16(b + L::AM_OFF + li * WS + 2 * (r - 16), a.Acoef + (size_t)l * Bp + m0 + 2 * (r - 16));
        }
        if (lc + LW_CH - 1 > blo) {
            for (int i = tid; i < LW_CH * (NP * 16 + WS); i += blockDim.x) {
                const int li = i / (NP * 16 + WS), r = i % (NP * 16 + WS), l = lc + li;
                if (l >= bl || l <= blo) continue;
                if (r < NP * 16) {
                    const int q = r >> 4, c2 = r & 15;
                    cp16(b + L::G_OFF + (li * NP + q) * 32 + 2 * c2,
                         a.G + ((size_t)(l - blo - 1) * NP + q) * Gs + p0 + 2 * c2);
                } else {
                    const int c1 = r - NP * 16;
                    cp16(b + L::F_OFF + 2 * (li * WS + c1), a.F + (size_t)l * Bp + m0 + c1);
                }
            }
        }
    };

    // One recurrence step at chunk row li (l parity PAR).
    auto step = [&](const double *b, const int li, const int l, auto par_tag, const bool inj, const bool accum) {
        constexpr int PAR = decltype(par_tag)::value;
        const double ap = b[L::AP_OFF + li * 32 + lane];
        double g[NP];
        if (accum) {
#pragma unroll
            for (int q = 0; q < NP; q++) g[q] = b[L::G_OFF + (li * NP + q) * 32 + lane];
        }
        const double2 *Fr = reinterpret_cast<const double2 *>(b + L::F_OFF) + li * WS + w * S;
        const double *Amr = b + L::AM_OFF + li * WS + w * S;
#pragma unroll
        for (int s = 0; s < S; s++) {
            if (inj && l == l0[s]) e[s] = st[s];
            if (accum) {
                const double2 F = Fr[s];
                const double xr = e[s] * F.x, xi = e[s] * F.y;
#pragma unroll
                for (int q = 0; q < NP; q++) {
                    acc[PAR][s][q].x = fma(xr, g[q], acc[PAR][s][q].x);
                    acc[PAR][s][q].y = fma(xi, g[q], acc[PAR][s][q].y);
                }
            }
            const double p = Amr[s] * ap;
            const double en = fma(-p, e[s], -ep[s]);
            ep[s] = e[s];
            e[s] = en;
        }
    };
    using P0 = std::integral_constant<int, 0>;
    using P1 = std::integral_constant<int, 1>;

    if (nchunks > 0) stage(0, 0);
    cp_commit();
    for (int c = 0; c < nchunks; c++) {
        if (c + 1 < nchunks) stage(c + 1, (c + 1) & 1);
        cp_commit();
        cp_wait<1>();
        __syncthreads();
        const double *b = lsm + (c & 1) * L::BUF;
        const int lc = lstart + c * LW_CH;
        const int nl = min(LW_CH, bl - lc);
        if (lc > rampEnd && lc > blo && nl == LW_CH) {
#pragma unroll 1
            for (int li = 0; li < LW_CH; li += 2) {
                step(b, li, lc + li, P0{}, false, true);
                step(b, li + 1, lc + li + 1, P1{}, false, true);
            }
        } else {
#pragma unroll 1
            for (int li = 0; li < nl; li += 2) {
                const int l = lc + li;
                step(b, li, l, P0{}, l <= rampEnd, l > blo);
                if (li + 1 < nl) step(b, li + 1, l + 1, P1{}, l + 1 <= rampEnd, l + 1 > blo);
            }
        }
        if (Kw > 0) {  // keep scaled values in range (warp-uniform)
            double mx = 0.0;
#pragma unroll
            for (int s = 0; s < S; s++) mx = fmax(mx, fmax(fabs(e[s]), fabs(ep[s])));
            mx = warp_max(mx);
            if (mx > ldexp(1.0, S2DW_RENORM_EXP)) {
                const int R = min(S2DW_RENORM_EXP, Kw);
                const double f = ldexp(1.0, -R);
#pragma unroll
                for (int s = 0; s < S; s++) {
                    e[s] *= f;
                    ep[s] *= f;
#pragma unroll
                    for (int q = 0; q < NP; q++) {
                        acc[0][s][q] = cscale(acc[0][s][q], f);
                        acc[1][s][q] = cscale(acc[1][s][q], f);
                    }
                }
                Kw -= R;
            }
        }
        __syncthreads();
    }

    // ---- epilogue: T(m,m',+-n) from even/odd-l sums, then the gamma DFT
    // T(+n) = i^{n-m} conj(eta) (E+O), T(-n) = i^{-n-m} (-1)^{m'+n} eta (E-O),
    // T(0) = i^{-m} (E+O); eta = 1 (N odd) or i (N even).
    const double sc = ldexp(1.0, -Kw);
    const int ev = (N % 2 == 0) ? 1 : 0;
#pragma unroll
    for (int s = 0; s < S; s++) {
        if (l0[s] == INT_MAX) continue;
        const int m = m0 + w * S + s;
        double2 Tp[NP], Tm[NP];
#pragma unroll
        for (int q = 0; q < NP; q++) {
            const int n = a.nq[q];
            const double2 E = cscale(acc[0][s][q], sc), O = cscale(acc[1][s][q], sc);
            const double2 sum = cadd(E, O), dif = csub(E, O);
            if (n == 0) {
                Tp[q] = cipow(sum, -m);
                Tm[q] = make_double2(0.0, 0.0);
            } else {
                Tp[q] = cipow(sum, n - m - ev);
                double2 t = cipow(dif, -n - m + ev);
                if ((mp + n) & 1) t = make_double2(-t.x, -t.y);
                Tm[q] = t;
            }
        }
        for (int gg = 0; gg < N; gg++) {
            double2 y = make_double2(0.0, 0.0);
#pragma unroll
            for (int q = 0; q < NP; q++) {
                const int n = a.nq[q];
                y = cadd(y, cmul(Tp[q], sPh[gg * 16 + n + N - 1]));
                if (n != 0) y = cadd(y, cmul(Tm[q], sPh[gg * 16 - n + N - 1]));
            }
            a.Tg[((size_t)gg * bl + m) * bl + mp] = y;
        }
    }
}

// Per-scale factor tables for the contraction kernels (built once per set of
// kernel tables).
__global__ void gprep_kernel(GprepArgs a)
{
    const int nl = a.bl - a.blo - 1;
    const long long total = (long long)nl * a.NP * a.stride;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % a.stride);
        const long long r = i / a.stride;
        const int q = (int)(r % a.NP), l = a.blo + 1 + (int)(r / a.NP);
        double v = 0.0;
        if (x <= l && x < a.bl)
            v = a.T[(size_t)l * a.Bp + x] * a.H[((size_t)l * 8 + a.nq[q]) * a.B + x] * a.kappa[(size_t)l * a.NP + q];
        a.out[i] = v;
    }
}

// F[l*Bp + m] = Om[l*Bp+m] flm[l + B m]: transpose of the column-major flm
// through a 32x32 shared tile.
__global__ void fprep_kernel(double2 *F, const double2 *flm, const double *Om, int B, int Bp)
{
    __shared__ double2 tile[32][33];
    const int l0 = blockIdx.x * 32, mb = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (int k = ty; k < 32; k += 8) {
        const int l = l0 + tx, m = mb + k;
        tile[k][tx] = (l < B && m < B) ? flm[(size_t)l + (size_t)B * m] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
        const int l = l0 + k, m = mb + tx;
        if (l < B && m < Bp) {
            double2 v = make_double2(0.0, 0.0);
            if (m <= l && m < B) v = cscale(tile[tx][k], Om[(size_t)l * Bp + m]);
            F[(size_t)l * Bp + m] = v;
        }
    }
}

// ===========================================================================
// Synthesis: m'-walk contraction and harmonic accumulation
//
// CTA tile: 32 consecutive l (lanes) x MW_W*Q consecutive m (Q per warp).
// Each thread walks m' down from min(l_tile_max, bl-1) to 0 for its Q pairs
// (l, m).  Staged per chunk of MW_CH m' values (aligned to MW_CH): the
// lane-distinct rows b(l, m') and G(l, m', q) (each thread copies its row to
// registers) and the broadcast V2f(m, m', q).
// ===========================================================================
constexpr int MW_W = 4;
constexpr int MW_CH = 8;
constexpr int MW_RS = MW_CH + 2;  // padded row stride (conflict-free 16-byte row loads)

template <int NP, int Q>
struct MwalkSmem {
    static constexpr int WQ = MW_W * Q;
    static constexpr int V_OFF = 0;                          // double2 [NP][WQ][MW_CH]
    static constexpr int B_OFF = V_OFF + 2 * NP * WQ * MW_CH;  // double [32][MW_RS]
    static constexpr int G_OFF = B_OFF + 32 * MW_RS;           // double [NP][32][MW_RS]
    static constexpr int BUF = G_OFF + NP * 32 * MW_RS;
    static constexpr size_t BYTES = 2 * BUF * sizeof(double);
};

template <int NP, int Q>
__global__ void __launch_bounds__(MW_W * 32) mwalk_kernel(MwalkArgs a, int tiles_m)
{
    using L = MwalkSmem<NP, Q>;
    constexpr int WQ = L::WQ;
    extern __shared__ __align__(16) double msm[];

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int mt = blockIdx.x % tiles_m, lt = blockIdx.x / tiles_m;
    const int B = a.B, Bp = a.Bp, bl = a.bl, blo = a.blo, Gs = a.Gs, Vs = a.Vs;
    const int lbase = blo + 1 + lt * 32, mbase = mt * WQ;
    const int MH = min(lbase + 31, bl - 1);
    if (mbase > MH) return;  // tile entirely above the diagonal m <= l
    const int l = lbase + lane;

    double st[Q], mq[Q];
    bool val[Q];
    int maxe = INT_MIN;
#pragma unroll
    for (int q = 0; q < Q; q++) {
        const int m = mbase + w * Q + q;
        val[q] = (l < bl) && (m <= l);
        mq[q] = (double)m;
        if (val[q]) maxe = max(maxe, (int)a.Ee[(size_t)l * B + m]);
    }
    maxe = warp_max_i(maxe);
    int Kw = (maxe != INT_MIN && maxe < S2DW_SCALE_EXP) ? -maxe : 0;
#pragma unroll
    for (int q = 0; q < Q; q++) {
        const int m = mbase + w * Q + q;
        st[q] = 0.0;
        if (val[q]) {
            const double v = ldexp(a.Em[(size_t)l * B + m], (int)a.Ee[(size_t)l * B + m] + Kw);
            st[q] = ((l - m) & 1) ? -v : v;
        }
    }
    double e[Q], ep[Q];
    double2 acc[Q];
#pragma unroll
    for (int q = 0; q < Q; q++) {
        e[q] = ep[q] = 0.0;
        acc[q] = make_double2(0.0, 0.0);
    }

    const int ctop = MH / MW_CH;  // chunks ctop, ctop-1, ..., 0 cover m' = MH .. 0

    auto stage = [&](int c, int buf) {
        double *b = msm + buf * L::BUF;
        const int c0 = c * MW_CH;
        // rows of b(l, m') and G(l, m', q): MW_CH/2 copies per row
        for (int i = tid; i < (1 + NP) * 32 * (MW_CH / 2); i += blockDim.x) {
            const int k = i % (MW_CH / 2), row = i / (MW_CH / 2), t = row % 32, q = row / 32;
            const int ll = lbase + t;
            double *dst = (q == 0) ? b + L::B_OFF + t * MW_RS + 2 * k
                                   : b + L::G_OFF + ((q - 1) * 32 + t) * MW_RS + 2 * k;
            if (ll < bl) {
                const double *src = (q == 0) ? a.Bcoef + (size_t)ll * Bp + c0 + 2 * k
                                             : a.G + ((size_t)(ll - blo - 1) * NP + (q - 1)) * Gs + c0 + 2 * k;
                cp16(dst, src);
            } else {
                dst[0] = 0.0;
                dst[1] = 0.0;
            }
        }
        // V2f(m, m', q) for the tile's m: MW_CH complex per (q, m)
        for (int i = tid; i < NP * WQ * MW_CH; i += blockDim.x) {
            const int k = i % MW_CH, r = i / MW_CH, u = r % WQ, q = r / WQ;
            const int m = mbase + u;
            double *dst = b + L::V_OFF + 2 * ((q * WQ + u) * MW_CH + k);
            if (m < bl) cp16(dst, a.V2f + ((size_t)q * bl + m) * Vs + c0 + k);
            else { dst[0] = 0.0; dst[1] = 0.0; }
        }
    };

    stage(ctop, 0);
    cp_commit();
    for (int c = ctop, it = 0; c >= 0; c--, it++) {
        if (c > 0) stage(c - 1, (it + 1) & 1);
        cp_commit();
        cp_wait<1>();
        __syncthreads();
        const double *b = msm + (it & 1) * L::BUF;
        const int c0 = c * MW_CH;
        // this thread's rows into registers
        double br[MW_CH], gr[NP][MW_CH];
#pragma unroll
        for (int k = 0; k < MW_CH; k += 2) {
            const double2 v = *reinterpret_cast<const double2 *>(b + L::B_OFF + lane * MW_RS + k);
            br[k] = v.x;
            br[k + 1] = v.y;
#pragma unroll
            for (int q = 0; q < NP; q++) {
                const double2 u = *reinterpret_cast<const double2 *>(b + L::G_OFF + (q * 32 + lane) * MW_RS + k);
                gr[q][k] = u.x;
                gr[q][k + 1] = u.y;
            }
        }
        const double2 *Vb = reinterpret_cast<const double2 *>(b + L::V_OFF);
        const bool ramp = (c0 + MW_CH - 1 >= lbase);
#pragma unroll
        for (int k = MW_CH - 1; k >= 0; k--) {
            const int mpv = c0 + k;
            if (mpv > MH) continue;  // above the top of this tile (warp-uniform)
#pragma unroll
            for (int q = 0; q < Q; q++) {
                if (ramp && mpv == l) e[q] = st[q];
                double zr = 0.0, zi = 0.0;
#pragma unroll
                for (int kq = 0; kq < NP; kq++) {
                    const double2 v = Vb[(kq * WQ + w * Q + q) * MW_CH + k];
                    zr = fma(gr[kq][k], v.x, zr);
                    zi = fma(gr[kq][k], v.y, zi);
                }
                acc[q].x = fma(e[q], zr, acc[q].x);
                acc[q].y = fma(e[q], zi, acc[q].y);
                const double p = mq[q] * br[k];
                const double en = fma(p, e[q], -ep[q]);
                ep[q] = e[q];
                e[q] = en;
            }
        }
        if (Kw > 0) {
            double mx = 0.0;
#pragma unroll
            for (int q = 0; q < Q; q++) mx = fmax(mx, fmax(fabs(e[q]), fabs(ep[q])));
            mx = warp_max(mx);
            if (mx > ldexp(1.0, S2DW_RENORM_EXP)) {
                const int R = min(S2DW_RENORM_EXP, Kw);
                const double f = ldexp(1.0, -R);
#pragma unroll
                for (int q = 0; q < Q; q++) {
                    e[q] *= f;
                    ep[q] *= f;
                    acc[q] = cscale(acc[q], f);
                }
                Kw -= R;
            }
        }
        __syncthreads();
    }
    // flm(l,m) += i^m * acc (the eta and i^{-n} phases are folded into G)
    const double sc = ldexp(1.0, -Kw);
#pragma unroll
    for (int q = 0; q < Q; q++) {
        if (!val[q]) continue;
        const int m = mbase + w * Q + q;
        double2 *f = a.flm + (size_t)l + (size_t)B * m;
        *f = cadd(*f, cipow(cscale(acc[q], sc), m));
    }
}

// ===========================================================================
// Chirp-z transform engine: power-of-two FFTs in shared memory
// ===========================================================================

// exp(SIGN * 2 pi i k / 16) for k in [0, 8)
template <int SIGN>
__device__ __forceinline__ double2 w16(int k)
{
    const double C[8] = {1.0, 0.92387953251128675613, 0.70710678118654752440, 0.38268343236508977173,
                         0.0, -0.38268343236508977173, -0.70710678118654752440, -0.92387953251128675613};
    const double Sn[8] = {0.0, 0.38268343236508977173, 0.70710678118654752440, 0.92387953251128675613,
                          1.0, 0.92387953251128675613, 0.70710678118654752440, 0.38268343236508977173};
    return make_double2(C[k], SIGN * Sn[k]);
}

// In-register DFT of size R (R = 1, 2, 4, 8, 16), radix-2 decimation in time.
template <int R, int SIGN>
struct Dft {
    __device__ __forceinline__ static void run(double2 *v)
    {
        double2 ev[R / 2], od[R / 2];
#pragma unroll
        for (int i = 0; i < R / 2; i++) {
            ev[i] = v[2 * i];
            od[i] = v[2 * i + 1];
        }
        Dft<R / 2, SIGN>::run(ev);
        Dft<R / 2, SIGN>::run(od);
#pragma unroll
        for (int k = 0; k < R / 2; k++) {
            double2 t;
            if (k == 0) t = od[k];
            else if (4 * k == R) t = (SIGN < 0) ? make_double2(od[k].y, -od[k].x) : make_double2(-od[k].y, od[k].x);
            else t = cmul(od[k], w16<SIGN>(k * (16 / R)));
            v[k] = cadd(ev[k], t);
            v[k + R / 2] = csub(ev[k], t);
        }
    }
};
template <int SIGN>
struct Dft<1, SIGN> {
    __device__ __forceinline__ static void run(double2 *) {}
};

__host__ __device__ __forceinline__ int padix(int i) { return i + (i >> 4); }

// W_M^x (forward) from the two-level tables.
__device__ __forceinline__ double2 twid(const double2 *twh, const double2 *twl, int x)
{
    return cmul(twh[x >> 6], twl[x & 63]);
}

// One Stockham pass of radix R over `rows` transforms of size M held at
// buf[r*M ...] (padded indices).  Each thread processes NB = 16/R butterflies.
template <int R, int SIGN>
__device__ __forceinline__ void fft_pass(double2 *buf, int M, int Ns, int tid,
                                         const double2 *twh, const double2 *twl)
{
    constexpr int NB = 16 / R;
    const int perRow = M / R;
    double2 v[NB][R];
    int base[NB], jj[NB];
#pragma unroll
    for (int u = 0; u < NB; u++) {
        const int b = tid * NB + u, r = b / perRow, j = b % perRow;
        base[u] = r * M;
        jj[u] = j;
#pragma unroll
        for (int t = 0; t < R; t++) v[u][t] = buf[padix(base[u] + j + t * perRow)];
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < NB; u++) {
        const int j = jj[u], k = j % Ns;
        const int step = k * (M / (Ns * R));
#pragma unroll
        for (int t = 1; t < R; t++) {
            double2 wv = twid(twh, twl, step * t);
            if (SIGN > 0) wv = cconj(wv);
            v[u][t] = cmul(v[u][t], wv);
        }
        Dft<R, SIGN>::run(v[u]);
        const int idx = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int t = 0; t < R; t++) buf[padix(base[u] + idx + t * Ns)] = v[u][t];
    }
    __syncthreads();
}

template <int SIGN>
__device__ void fft_rows(double2 *buf, int M, int tid, const double2 *twh, const double2 *twl)
{
    int Ns = 1;
    while (Ns * 16 <= M) {
        fft_pass<16, SIGN>(buf, M, Ns, tid, twh, twl);
        Ns *= 16;
    }
    const int rem = M / Ns;
    if (rem == 2) fft_pass<2, SIGN>(buf, M, Ns, tid, twh, twl);
    else if (rem == 4) fft_pass<4, SIGN>(buf, M, Ns, tid, twh, twl);
    else if (rem == 8) fft_pass<8, SIGN>(buf, M, Ns, tid, twh, twl);
}

// rows per CTA so that every CTA holds max(M, 4096) complex values
__host__ __device__ __forceinline__ int czt_elems(int M) { return M > 4096 ? M : 4096; }

__global__ void __launch_bounds__(512) czt_kernel(CztArgs a)
{
    extern __shared__ double2 smem[];
    const int M = a.czt.M, E = czt_elems(M), R = E / M;
    double2 *buf = smem;
    double2 *twh = smem + padix(E) + 1;
    const int nhi = (M + 63) / 64;
    double2 *twl = twh + nhi;
    double2 *ph = twl + 64;  // [q][g] exp(-i pi n_q g / N) for CZT_SYN_BETA
    const int tid = threadIdx.x, T = blockDim.x;
    const int bl = a.bl, n = 2 * bl - 1, N = a.N, K = a.czt.spec.K, Bout = a.czt.spec.Bout;
    const int row0 = blockIdx.x * R;

    for (int i = tid; i < nhi; i += T) twh[i] = a.tw.hi[i];
    for (int i = tid; i < 64; i += T) twl[i] = a.tw.lo[i];
    if (a.mode == CZT_SYN_BETA)
        for (int i = tid; i < a.NP * N; i += T) {
            const int q = i / N, g = i % N;
            double s, c;
            sincospi(-(double)(a.nq[q] * g) / (double)N, &s, &c);
            ph[i] = make_double2(c, s);
        }
    __syncthreads();

    // ---- load (with pre-chirp), zero padding to M
    for (int i = tid; i < E; i += T) {
        const int r = i / M, k = i % M, row = row0 + r;
        double2 x = make_double2(0.0, 0.0);
        if (row < a.rows && k < K) {
            switch (a.mode) {
            case CZT_ANA_BETA: {  // row = (g, m); k <-> m' = k-(bl-1)
                const int g = row / bl, m = row % bl, mpv = k - (bl - 1), ab = mpv < 0 ? -mpv : mpv;
                x = a.in_c[((size_t)g * bl + m) * bl + ab];
                if (((m + N - 1) & 1) && mpv < 0) x = make_double2(-x.x, -x.y);
                break;
            }
            case CZT_ANA_ALPHA: {  // row = (g, b pair); Hermitian completion in m
                const int g = row / bl, bp = row % bl;
                const size_t base = (size_t)g * bl;
                double2 x1, x2;
                if (k < bl) {
                    const double2 *p = a.in_c + (base + k) * (2 * bl) + 2 * bp;
                    x1 = p[0];
                    x2 = p[1];
                    if (k == 0) { x1.y = 0.0; x2.y = 0.0; }
                } else {
                    const double2 *p = a.in_c + (base + (n - k)) * (2 * bl) + 2 * bp;
                    x1 = cconj(p[0]);
                    x2 = cconj(p[1]);
                }
                x = make_double2(x1.x - x2.y, x1.y + x2.x);
                break;
            }
            case CZT_SYN_ALPHA: {  // row = (g, b pair); z = w(:,b1) + i w(:,b2)
                const int g = row / bl, bp = row % bl;
                const double *p = a.in_r + (size_t)k + (size_t)n * (2 * bp + (size_t)2 * bl * g);
                x = make_double2(p[0], p[n]);
                break;
            }
            default: {  // CZT_SYN_BETA: row = (q, m); k = b; gamma DFT on the fly
                const int q = row / bl, m = row % bl;
                double2 u = make_double2(0.0, 0.0);
                for (int g = 0; g < N; g++)
                    u = cadd(u, cmul(a.in_c[((size_t)g * bl + m) * (2 * bl) + k], ph[q * N + g]));
                x = cscale(u, a.wq[k]);
                break;
            }
            }
            x = cmul(x, a.czt.pre[k]);
        }
        buf[padix(i)] = x;
    }
    __syncthreads();
    fft_rows<-1>(buf, M, tid, twh, twl);
    for (int i = tid; i < E; i += T) {
        const int k = i % M;
        buf[padix(i)] = cmul(buf[padix(i)], a.czt.Hf[k]);
    }
    __syncthreads();
    fft_rows<+1>(buf, M, tid, twh, twl);

    // ---- post-chirp and store
    switch (a.mode) {
    case CZT_ANA_BETA:
        for (int i = tid; i < R * Bout; i += T) {
            const int r = i / Bout, b = i % Bout, row = row0 + r;
            if (row >= a.rows) continue;
            const int g = row / bl, m = row % bl;
            a.out_c[((size_t)g * bl + m) * (2 * bl) + b] = cmul(buf[padix(r * M + b)], a.czt.post[b]);
        }
        break;
    case CZT_ANA_ALPHA:
        for (int i = tid; i < R * Bout; i += T) {
            const int r = i / Bout, aa = i % Bout, row = row0 + r;
            if (row >= a.rows) continue;
            const int g = row / bl, bp = row % bl;
            const double2 y = cmul(buf[padix(r * M + aa)], a.czt.post[aa]);
            double *p = a.out_r + (size_t)aa + (size_t)n * (2 * bp + (size_t)2 * bl * g);
            p[0] = y.x;
            p[n] = y.y;
        }
        break;
    case CZT_SYN_ALPHA:
        for (int i = tid; i < R * bl; i += T) {
            const int r = i / bl, m = i % bl, row = row0 + r;
            if (row >= a.rows) continue;
            const int g = row / bl, bp = row % bl;
            const int mc = (m == 0) ? 0 : n - m;
            const double2 Z = cmul(buf[padix(r * M + m)], a.czt.post[m]);
            const double2 Zc = cconj(cmul(buf[padix(r * M + mc)], a.czt.post[mc]));
            const double2 s = cadd(Z, Zc), d = csub(Z, Zc);
            const double h = 0.5 * a.scale;
            double2 *p = a.out_c + ((size_t)g * bl + m) * (2 * bl) + 2 * bp;
            p[0] = make_double2(s.x * h, s.y * h);
            p[1] = make_double2(d.y * h, -d.x * h);
        }
        break;
    default:  // CZT_SYN_BETA: fold +-m' and store V2f[q][m][m']
        for (int i = tid; i < R * bl; i += T) {
            const int r = i / bl, mpv = i % bl, row = row0 + r;
            if (row >= a.rows) continue;
            const int q = row / bl, m = row % bl;
            const int t0 = bl - 1 + mpv;
            double2 y = cmul(buf[padix(r * M + t0)], a.czt.post[t0]);
            if (mpv > 0) {
                const int t1 = bl - 1 - mpv;
                double2 z = cmul(buf[padix(r * M + t1)], a.czt.post[t1]);
                if ((m + a.nq[q]) & 1) z = make_double2(-z.x, -z.y);
                y = cadd(y, z);
            }
            a.out_c[((size_t)q * bl + m) * a.out_stride + mpv] = y;
        }
        break;
    }
}

// ===========================================================================
// Small kernels
// ===========================================================================
__global__ void zero_kernel(double *p, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = 0.0;
}

// scoeff(0:bs-1,0:bs-1) = flm(0:bs-1,0:bs-1), s2dw_core_mod.f90:773
__global__ void scoeff_copy_kernel(double2 *sc, const double2 *flm, int B, int bs)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < bs * bs) sc[i] = flm[(i % bs) + (size_t)B * (i / bs)];
}

// flm(l,0:bs-1) += Phi2(l) scoeff(l,0:bs-1), s2dw_core_mod.f90:1258-1261
__global__ void scaling_add_kernel(double2 *flm, const double2 *sc, const double *Phi2, int B, int bs)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < bs * bs) {
        const int l = i % bs, m = i / bs;
        double2 *f = flm + l + (size_t)B * m;
        *f = cadd(*f, cscale(sc[i], Phi2[l]));
    }
}

// ===========================================================================
// Launchers
// ===========================================================================
template <int NP, int S>
static int launch_lwalk_np(const LwalkArgs &a, cudaStream_t s)
{
    using L = LwalkSmem<NP, S>;
    static bool attr[64] = {false};
    int dev = 0;
    S2DW_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 64 && !attr[dev]) {
        S2DW_CUDA_TRY(cudaFuncSetAttribute(lwalk_kernel<NP, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)L::BYTES));
        attr[dev] = true;
    }
    const int tiles_p = (a.bl + 31) / 32, tiles_m = (a.bl + L::WS - 1) / L::WS;
    lwalk_kernel<NP, S><<<tiles_p * tiles_m, LW_W * 32, L::BYTES, s>>>(a, tiles_p);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

int launch_lwalk(const LwalkArgs &a, cudaStream_t s)
{
    switch (a.NP) {
    case 1: return launch_lwalk_np<1, 4>(a, s);
    case 2: return launch_lwalk_np<2, 4>(a, s);
    case 3: return launch_lwalk_np<3, 4>(a, s);
    case 4: return launch_lwalk_np<4, 4>(a, s);
    }
    return set_error(S2DWC_ERROR_SIZE_INVALID, "lwalk: unsupported N=%d (N<=8)", a.N);
}

template <int NP, int Q>
static int launch_mwalk_np(const MwalkArgs &a, cudaStream_t s)
{
    using L = MwalkSmem<NP, Q>;
    const int nl = a.bl - a.blo - 1;
    if (nl <= 0) return S2DWC_OK;
    static bool attr[64] = {false};
    int dev = 0;
    S2DW_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 64 && !attr[dev]) {
        S2DW_CUDA_TRY(cudaFuncSetAttribute(mwalk_kernel<NP, Q>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)L::BYTES));
        attr[dev] = true;
    }
    const int tiles_l = (nl + 31) / 32, tiles_m = (a.bl + L::WQ - 1) / L::WQ;
    mwalk_kernel<NP, Q><<<tiles_l * tiles_m, MW_W * 32, L::BYTES, s>>>(a, tiles_m);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

int launch_mwalk(const MwalkArgs &a, cudaStream_t s)
{
    switch (a.NP) {
    case 1: return launch_mwalk_np<1, 8>(a, s);
    case 2: return launch_mwalk_np<2, 8>(a, s);
    case 3: return launch_mwalk_np<3, 8>(a, s);
    case 4: return launch_mwalk_np<4, 8>(a, s);
    }
    return set_error(S2DWC_ERROR_SIZE_INVALID, "mwalk: unsupported N=%d (N<=8)", a.N);
}

int launch_gprep(const GprepArgs &a, cudaStream_t s)
{
    const long long total = (long long)(a.bl - a.blo - 1) * a.NP * a.stride;
    if (total <= 0) return S2DWC_OK;
    long long blocks = (total + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    gprep_kernel<<<(int)blocks, 256, 0, s>>>(a);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

int launch_fprep(double2 *F, const double2 *flm, const double *Om, int B, int Bp, cudaStream_t s)
{
    dim3 grid((B + 31) / 32, (Bp + 31) / 32), block(32, 8);
    fprep_kernel<<<grid, block, 0, s>>>(F, flm, Om, B, Bp);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

int launch_czt(const CztArgs &a, cudaStream_t s)
{
    const int M = a.czt.M, E = czt_elems(M), R = E / M;
    const int threads = E / 16;
    const int nhi = (M + 63) / 64;
    const size_t smem = sizeof(double2) * ((size_t)padix(E) + 1 + nhi + 64 + 32);
    static bool attr_set[64] = {false};
    int dev = 0;
    S2DW_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 64 && !attr_set[dev]) {
        S2DW_CUDA_TRY(cudaFuncSetAttribute(czt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           200 * 1024));
        attr_set[dev] = true;
    }
    const int grid = (a.rows + R - 1) / R;
    if (grid == 0) return S2DWC_OK;
    czt_kernel<<<grid, threads, smem, s>>>(a);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

int launch_zero(double *p, long long n, cudaStream_t s)
{
    if (n <= 0) return S2DWC_OK;
    long long blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    zero_kernel<<<(int)blocks, 256, 0, s>>>(p, n);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

int launch_scoeff_copy(double2 *scoeff, const double2 *flm, int B, int bs, cudaStream_t s)
{
    const int n = bs * bs;
    if (n <= 0) return S2DWC_OK;
    scoeff_copy_kernel<<<(n + 255) / 256, 256, 0, s>>>(scoeff, flm, B, bs);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

int launch_scaling_add(double2 *flm, const double2 *scoeff, const double *Phi2, int B, int bs,
                       cudaStream_t s)
{
    const int n = bs * bs;
    if (n <= 0) return S2DWC_OK;
    scaling_add_kernel<<<(n + 255) / 256, 256, 0, s>>>(flm, scoeff, Phi2, B, bs);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

}  // namespace s2dw
