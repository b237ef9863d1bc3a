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

#include <algorithm>
#include <climits>
#include <vector>
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
constexpr int LW_PHS = 2 * S2DW_NMAX;  // gamma-DFT phase table row: n + N - 1 < 2N - 1

template <int NP, int S>
struct LwalkSmem {
    static constexpr int WS = LW_W * S;
    // per buffer, in doubles: F (complex, first for 16-byte alignment), Ap, G, Am
    static constexpr int F_OFF = 0;
    static constexpr int AP_OFF = F_OFF + 2 * LW_CH * WS;
    static constexpr int G_OFF = AP_OFF + LW_CH * 32;
    static constexpr int AM_OFF = G_OFF + LW_CH * NP * 32;
    static constexpr int BUF = AM_OFF + LW_CH * WS;
    static constexpr size_t BYTES = 2 * BUF * sizeof(double) + S2DW_NMAX * LW_PHS * sizeof(double2);
};

template <int NP, int S>
__device__ __forceinline__ void lwalk_body(const LwalkArgs &a)
{
    using L = LwalkSmem<NP, S>;
    constexpr int WS = L::WS;
    extern __shared__ __align__(16) double lsm[];
    double2 *sPh = reinterpret_cast<double2 *>(lsm + 2 * L::BUF);  // [g*LW_PHS + n+N-1]

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int2 tile = a.tiles[blockIdx.x];
    const int p0 = tile.x * 32, m0 = tile.y * WS;
    const int B = a.B, Bp = a.Bp, bl = a.bl, blo = a.blo, N = a.N, Gs = a.Gs;
    const int mp = p0 + lane;

    for (int i = tid; i < N * (2 * N - 1); i += blockDim.x) {
        const int g = i / (2 * N - 1), n = i % (2 * N - 1) - (N - 1);
        double sn, cs;
        sincospi((double)(n * g) / (double)N, &sn, &cs);
        sPh[g * LW_PHS + n + N - 1] = make_double2(cs, sn);
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

    double x[2][S];
    double2 acc[2][S][NP];
#pragma unroll
    for (int s = 0; s < S; s++) {
        x[0][s] = 0.0;
        x[1][s] = 0.0;
#pragma unroll
        for (int q = 0; q < NP; q++) acc[0][s][q] = acc[1][s][q] = make_double2(0.0, 0.0);
    }

    const int lstart = max(p0, m0) & ~1;
    const int rampEnd = min(max(p0 + 31, m0 + WS - 1), bl - 1);
    const int nchunks = (bl - lstart + LW_CH - 1) / LW_CH;

    // Staging: the 16-byte pieces of a chunk's rows go to the threads in a
    // fixed pattern (piece column from the thread index, rows in passes), so
    // that a copy costs a row bound check and one address computation.
    static_assert(LW_W * 32 == 128 && LW_CH % 8 == 0, "staging pattern assumes 128 threads");
    auto stage = [&](int c, int buf) {
        const int lc = lstart + c * LW_CH;
        double *b = lsm + buf * L::BUF;
        const int pc = tid & 15;  // piece of a 32-double row
        // a(l, m'): 16 pieces per row, 8 rows per pass
#pragma unroll
        for (int i = 0; i < LW_CH / 8; i++) {
            const int li = (tid >> 4) + 8 * i, l = lc + li;
            if (l < bl) cp16(b + L::AP_OFF + li * 32 + 2 * pc, a.Acoef + (size_t)l * Bp + p0 + 2 * pc);
        }
        // a(l, m): WS/2 pieces per row
        constexpr int AMP = WS / 2, AMR = 128 / AMP;
#pragma unroll
        for (int i = 0; i < (LW_CH + AMR - 1) / AMR; i++) {
            const int li = tid / AMP + AMR * i, l = lc + li;
            if (li < LW_CH && l < bl)
                cp16(b + L::AM_OFF + li * WS + 2 * (tid % AMP), a.Acoef + (size_t)l * Bp + m0 + 2 * (tid % AMP));
        }
        if (lc + LW_CH - 1 > blo) {
            // G(l, m', q): rows r = li NP + q of 16 pieces, 8 rows per pass
#pragma unroll
            for (int i = 0; i < LW_CH * NP / 8; i++) {
                const int r = (tid >> 4) + 8 * i, l = lc + r / NP;
                if (l > blo && l < bl)
                    cp16(b + L::G_OFF + r * 32 + 2 * pc,
                         a.G + ((long long)(lc - blo - 1) * NP + r) * Gs + p0 + 2 * pc);
            }
            // F(l, m): WS pieces (complex values) per row
            constexpr int FR = 128 / WS;
#pragma unroll
            for (int i = 0; i < (LW_CH + FR - 1) / FR; i++) {
                const int li = tid / WS + FR * i, l = lc + li;
                if (li < LW_CH && l > blo && l < bl)
                    cp16(b + L::F_OFF + 2 * (li * WS + tid % WS), a.F + (size_t)l * Bp + m0 + tid % WS);
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
            if (inj && l == l0[s]) x[PAR][s] = st[s];
            const double cur = x[PAR][s];
            if (accum) {
                const double2 F = Fr[s];
                const double xr = cur * F.x, xi = cur * F.y;
#pragma unroll
                for (int q = 0; q < NP; q++) {
                    acc[PAR][s][q].x = fma(xr, g[q], acc[PAR][s][q].x);
                    acc[PAR][s][q].y = fma(xi, g[q], acc[PAR][s][q].y);
                }
            }
            const double p = Amr[s] * ap;
            x[PAR ^ 1][s] = fma(-p, cur, -x[PAR ^ 1][s]);
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
            // every step accumulates, no start value enters: unrolled, so that
            // the shared-memory reads take constant offsets
#pragma unroll
            for (int li = 0; li < LW_CH; li += 2) {
                step(b, li, lc + li, P0{}, false, true);
                step(b, li + 1, lc + li + 1, P1{}, false, true);
            }
        } else if (lc > rampEnd && lc + LW_CH - 1 <= blo && nl == LW_CH) {
            // a chunk below the scale's l range: the recurrence alone (not the
            // general path below, whose accumulation would issue predicated off)
#pragma unroll 1
            for (int li = 0; li < LW_CH; li += 2) {
                step(b, li, lc + li, P0{}, false, false);
                step(b, li + 1, lc + li + 1, P1{}, false, false);
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
            for (int s = 0; s < S; s++) mx = fmax(mx, fmax(fabs(x[0][s]), fabs(x[1][s])));
            mx = warp_max(mx);
            if (mx > ldexp(1.0, S2DW_RENORM_EXP)) {
                const int R = min(S2DW_RENORM_EXP, Kw);
                const double f = ldexp(1.0, -R);
#pragma unroll
                for (int s = 0; s < S; s++) {
                    x[0][s] *= f;
                    x[1][s] *= f;
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
            // acc_imag: the b part of S enters the +n terms times -i (i^-1)
            // and the -n terms times +i
            const int ai = a.acc_imag ? 1 : 0;
            if (n == 0) {
                Tp[q] = cipow(sum, -m - ai);
                Tm[q] = make_double2(0.0, 0.0);
            } else {
                Tp[q] = cipow(sum, n - m - ev - ai);
                double2 t = cipow(dif, -n - m + ev + ai);
                if ((mp + n) & 1) t = make_double2(-t.x, -t.y);
                Tm[q] = t;
            }
        }
        for (int gg = 0; gg < N; gg++) {
            double2 y = make_double2(0.0, 0.0);
#pragma unroll
            for (int q = 0; q < NP; q++) {
                const int n = a.nq[q];
                y = cadd(y, cmul(Tp[q], sPh[gg * LW_PHS + n + N - 1]));
                if (n != 0) y = cadd(y, cmul(Tm[q], sPh[gg * LW_PHS - n + N - 1]));
            }
            double2 *dst = a.Tg + ((size_t)gg * bl + m) * bl + mp;
            *dst = a.acc_imag ? cadd(*dst, y) : y;
        }
    }
}

// MINB = 0: no minimum-blocks bound (the compiler picks the register count)
template <int NP, int S, int MINB>
__global__ void __launch_bounds__(LW_W * 32) lwalk_kernel(LwalkArgs a)
{
    lwalk_body<NP, S>(a);
}
template <int NP, int S, int MINB>
__global__ void __launch_bounds__(LW_W * 32, MINB) lwalk_kernel_minb(LwalkArgs a)
{
    lwalk_body<NP, S>(a);
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
            v = a.T[(size_t)l * a.Bp + x] * a.H[((size_t)l * a.hn + a.nq[q]) * a.B + x] * a.kappa[(size_t)l * a.NP + q];
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
__device__ __forceinline__ void mwalk_body(const MwalkArgs &a)
{
    using L = MwalkSmem<NP, Q>;
    constexpr int WQ = L::WQ;
    extern __shared__ __align__(16) double msm[];

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int2 tile = a.tiles[blockIdx.x];
    const int lt = tile.x, mt = tile.y;
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

    // Staging: a fixed pattern of 16-byte pieces per thread (see lwalk).  The
    // rows of l >= bl and of m >= bl are never copied: they are zeroed once
    // here, in both buffers, so that the idle lanes and pairs walk zeros.
    static_assert(MW_W * 32 == 128 && MW_CH == 8, "staging pattern assumes 128 threads, 8 m' per chunk");
    const int nt = min(32, bl - lbase), nu = min(WQ, bl - mbase);
    if (nt < 32 || nu < WQ) {
        for (int i = tid; i < 2 * L::BUF; i += blockDim.x) {
            const int r = i % L::BUF;
            bool idle;
            if (r < L::B_OFF) idle = ((r - L::V_OFF) / (2 * MW_CH)) % WQ >= nu;
            else if (r < L::G_OFF) idle = (r - L::B_OFF) / MW_RS >= nt;
            else idle = ((r - L::G_OFF) / MW_RS) % 32 >= nt;
            if (idle) msm[i] = 0.0;
        }
    }
    auto stage = [&](int c, int buf) {
        double *b = msm + buf * L::BUF;
        const int c0 = c * MW_CH;
        // b(l, m') and G(l, m', q): 4 pieces per row, one row per 4 threads
        const int t = tid >> 2, k = tid & 3, ll = lbase + t;
        if (ll < bl) {
            cp16(b + L::B_OFF + t * MW_RS + 2 * k, a.Bcoef + (size_t)ll * Bp + c0 + 2 * k);
#pragma unroll
            for (int q = 0; q < NP; q++)
                cp16(b + L::G_OFF + (q * 32 + t) * MW_RS + 2 * k,
                     a.G + ((size_t)(ll - blo - 1) * NP + q) * Gs + c0 + 2 * k);
        }
        // V2f(m, m', q): MW_CH pieces (complex values) per (q, m) row
#pragma unroll
        for (int i = 0; i < NP * WQ * MW_CH / 128; i++) {
            const int f = tid + 128 * i, kk = f % MW_CH, r = f / MW_CH, u = r % WQ, q = r / WQ;
            if (mbase + u < bl)
                cp16(b + L::V_OFF + 2 * (r * MW_CH + kk), a.V2f + ((size_t)q * bl + mbase + u) * Vs + c0 + kk);
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
        // one step of the m' walk for pair q at chunk row k (the same
        // operations in the same order on both paths below)
        auto mstep = [&](const int k, const int q) {
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
        };
        if (!ramp && c0 + MW_CH - 1 <= MH) {
            // a chunk below the tile's l rows: every step runs, no start value
            // enters (warp-uniform)
#pragma unroll
            for (int k = MW_CH - 1; k >= 0; k--)
#pragma unroll
                for (int q = 0; q < Q; q++) mstep(k, q);
        } else {
#pragma unroll
            for (int k = MW_CH - 1; k >= 0; k--) {
                const int mpv = c0 + k;
                if (mpv > MH) continue;  // above the top of this tile (warp-uniform)
#pragma unroll
                for (int q = 0; q < Q; q++) {
                    if (ramp && mpv == l) e[q] = st[q];
                    mstep(k, q);
                }
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
    // this scale's flm(l,m) = i^m * acc (the eta and i^{-n} phases are folded into G)
    const double sc = ldexp(1.0, -Kw);
#pragma unroll
    for (int q = 0; q < Q; q++) {
        if (!val[q]) continue;
        const int m = mbase + w * Q + q;
        double2 *dst = a.part + (size_t)(l - blo - 1) * bl + m;
        if (a.acc_imag) *dst = cadd(*dst, cipow(cscale(acc[q], sc), m + 1));  // + i * result
        else *dst = cipow(cscale(acc[q], sc), m);
    }
}

template <int NP, int Q, int MINB>
__global__ void __launch_bounds__(MW_W * 32) mwalk_kernel(MwalkArgs a)
{
    mwalk_body<NP, Q>(a);
}
template <int NP, int Q, int MINB>
__global__ void __launch_bounds__(MW_W * 32, MINB) mwalk_kernel_minb(MwalkArgs a)
{
    mwalk_body<NP, Q>(a);
}

// ---------------------------------------------------------------------------
// Synthesis m'-walk with two l per thread (NP <= 4).
//
// The broadcast reads of V2f(m, m', q) bound the kernel above: a 16-byte read
// that every lane takes costs two shared-memory wavefronts, one per (m, q, m')
// for 32 lanes' worth of FP64 work.  Here each lane walks the pairs of two l
// (l and l + 32) with QM values of m, so that one broadcast read of V feeds
// twice the work, and the per-l rows b(l, m') and G(l, m', q) are read per step
// from a transposed table (GT, l fastest: conflict-free 8-byte reads) instead
// of being held in registers.  Tile: 64 l x MW_W*QM m; the same chunks of
// MW_CH m' values, staged by cp.async in a fixed pattern.
// ---------------------------------------------------------------------------
constexpr int M2_TL = 64;  // l per tile

template <int NP, int QM>
struct Mwalk2Smem {
    static constexpr int WQ = MW_W * QM;
    static constexpr int R = NP + 1;                               // GT rows per m'
    static constexpr int T_OFF = 0;                                // double [MW_CH][R][64]
    static constexpr int V_OFF = T_OFF + MW_CH * R * M2_TL;        // double2 [NP][WQ][MW_CH]
    static constexpr int BUF = V_OFF + 2 * NP * WQ * MW_CH;
    static constexpr size_t BYTES = 2 * BUF * sizeof(double);
};

template <int NP, int QM>
__device__ __forceinline__ void mwalk2_body(const MwalkArgs &a)
{
    using L = Mwalk2Smem<NP, QM>;
    constexpr int WQ = L::WQ, R = L::R;
    static_assert(MW_W * 32 == 128 && MW_CH == 8 && (MW_CH * R * M2_TL / 2) % 128 == 0, "staging pattern");
    extern __shared__ __align__(16) double msm[];

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int2 tile = a.tiles[blockIdx.x];
    const int lt = tile.x, mt = tile.y;
    const int B = a.B, bl = a.bl, blo = a.blo, Vs = a.Vs, Ts = a.Ts;
    const int lbase = blo + 1 + lt * M2_TL, mbase = mt * WQ;
    const int MH = min(lbase + M2_TL - 1, bl - 1);
    if (mbase > MH) return;  // tile entirely above the diagonal m <= l

    int l[2];
    double st[2][QM], mq[QM];
    bool val[2][QM];
    int maxe = INT_MIN;
#pragma unroll
    for (int i = 0; i < 2; i++) {
        l[i] = lbase + lane + 32 * i;
#pragma unroll
        for (int q = 0; q < QM; q++) {
            const int m = mbase + w * QM + q;
            val[i][q] = (l[i] < bl) && (m <= l[i]);
            if (val[i][q]) maxe = max(maxe, (int)a.Ee[(size_t)l[i] * B + m]);
        }
    }
#pragma unroll
    for (int q = 0; q < QM; q++) mq[q] = (double)(mbase + w * QM + q);
    maxe = warp_max_i(maxe);
    int Kw = (maxe != INT_MIN && maxe < S2DW_SCALE_EXP) ? -maxe : 0;
    double e[2][QM], ep[2][QM];
    double2 acc[2][QM];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int q = 0; q < QM; q++) {
            const int m = mbase + w * QM + q;
            st[i][q] = 0.0;
            if (val[i][q]) {
                const double v = ldexp(a.Em[(size_t)l[i] * B + m], (int)a.Ee[(size_t)l[i] * B + m] + Kw);
                st[i][q] = ((l[i] - m) & 1) ? -v : v;
            }
            e[i][q] = ep[i][q] = 0.0;
            acc[i][q] = make_double2(0.0, 0.0);
        }

    const int ctop = MH / MW_CH;  // chunks ctop, ctop-1, ..., 0 cover m' = MH .. 0
    // V rows of m >= bl are never copied: zeroed once, in both buffers
    const int nu = min(WQ, bl - mbase);
    if (nu < WQ)
        for (int i = tid; i < 2 * L::BUF; i += blockDim.x) {
            const int r = i % L::BUF;
            if (r >= L::V_OFF && ((r - L::V_OFF) / (2 * MW_CH)) % WQ >= nu) msm[i] = 0.0;
        }
    // GT rows (m', q) of a chunk are consecutive: MW_CH*R rows of 64 doubles
    // from column lt*64 (16-byte pieces, 32 per row); V2f as in mwalk_kernel
    const double *gsrc = a.GT + (size_t)lt * M2_TL;
    auto stage = [&](int c, int buf) {
        double *b = msm + buf * L::BUF;
        const double *src = gsrc + (size_t)c * MW_CH * R * Ts;
#pragma unroll
        for (int i = 0; i < MW_CH * R * M2_TL / 2 / 128; i++) {
            const int pc = tid + 128 * i, row = pc >> 5, col = pc & 31;
            cp16(b + L::T_OFF + row * M2_TL + 2 * col, src + (size_t)row * Ts + 2 * col);
        }
        const int c0 = c * MW_CH;
#pragma unroll
        for (int i = 0; i < (NP * WQ * MW_CH + 127) / 128; i++) {
            const int f = tid + 128 * i, kk = f % MW_CH, r = f / MW_CH, u = r % WQ, q = r / WQ;
            if (f < NP * WQ * MW_CH && mbase + u < bl)
                cp16(b + L::V_OFF + 2 * (r * MW_CH + kk), a.V2f + ((size_t)q * bl + mbase + u) * Vs + c0 + kk);
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
        const double *T = b + L::T_OFF;
        const double2 *Vb = reinterpret_cast<const double2 *>(b + L::V_OFF);
        const int c0 = c * MW_CH;
        const bool ramp = (c0 + MW_CH - 1 >= lbase);
        // one m' step at chunk row k for all pairs (the same operations in the
        // same order as mwalk_kernel's step)
        auto mstep = [&](const int k, const bool inj, const int mpv) {
            double bk[2], gk[2][NP];
#pragma unroll
            for (int i = 0; i < 2; i++) {
                bk[i] = T[(k * R + NP) * M2_TL + lane + 32 * i];
#pragma unroll
                for (int kq = 0; kq < NP; kq++) gk[i][kq] = T[(k * R + kq) * M2_TL + lane + 32 * i];
            }
#pragma unroll
            for (int q = 0; q < QM; q++) {
                double2 v[NP];
#pragma unroll
                for (int kq = 0; kq < NP; kq++) v[kq] = Vb[(kq * WQ + w * QM + q) * MW_CH + k];
#pragma unroll
                for (int i = 0; i < 2; i++) {
                    if (inj && mpv == l[i]) e[i][q] = st[i][q];
                    double zr = 0.0, zi = 0.0;
#pragma unroll
                    for (int kq = 0; kq < NP; kq++) {
                        zr = fma(gk[i][kq], v[kq].x, zr);
                        zi = fma(gk[i][kq], v[kq].y, zi);
                    }
                    acc[i][q].x = fma(e[i][q], zr, acc[i][q].x);
                    acc[i][q].y = fma(e[i][q], zi, acc[i][q].y);
                    const double p = mq[q] * bk[i];
                    const double en = fma(p, e[i][q], -ep[i][q]);
                    ep[i][q] = e[i][q];
                    e[i][q] = en;
                }
            }
        };
        if (!ramp && c0 + MW_CH - 1 <= MH) {
            // below the tile's l rows: every step runs, no start value enters
#pragma unroll
            for (int k = MW_CH - 1; k >= 0; k--) mstep(k, false, 0);
        } else {
#pragma unroll 1
            for (int k = MW_CH - 1; k >= 0; k--) {
                const int mpv = c0 + k;
                if (mpv > MH) continue;  // above the top of this tile (warp-uniform)
                mstep(k, ramp, mpv);
            }
        }
        if (Kw > 0) {
            double mx = 0.0;
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int q = 0; q < QM; q++) mx = fmax(mx, fmax(fabs(e[i][q]), fabs(ep[i][q])));
            mx = warp_max(mx);
            if (mx > ldexp(1.0, S2DW_RENORM_EXP)) {
                const int Rr = min(S2DW_RENORM_EXP, Kw);
                const double f = ldexp(1.0, -Rr);
#pragma unroll
                for (int i = 0; i < 2; i++)
#pragma unroll
                    for (int q = 0; q < QM; q++) {
                        e[i][q] *= f;
                        ep[i][q] *= f;
                        acc[i][q] = cscale(acc[i][q], f);
                    }
                Kw -= Rr;
            }
        }
        __syncthreads();
    }
    const double sc = ldexp(1.0, -Kw);
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int q = 0; q < QM; q++) {
            if (!val[i][q]) continue;
            const int m = mbase + w * QM + q;
            double2 *dst = a.part + (size_t)(l[i] - blo - 1) * bl + m;
            if (a.acc_imag) *dst = cadd(*dst, cipow(cscale(acc[i][q], sc), m + 1));  // + i * result
            else *dst = cipow(cscale(acc[i][q], sc), m);
        }
}

template <int NP, int QM>
__global__ void __launch_bounds__(MW_W * 32, 3) mwalk2_kernel(MwalkArgs a)
{
    mwalk2_body<NP, QM>(a);
}

// GT[(m' (NP+1) + q) Ts + l'] from G (q < NP) and b(l, m') (q = NP), l = blo+1+l';
// zero for l' >= bl-blo-1 or m' >= bl.
__global__ void gsyn_t_kernel(GsTArgs a)
{
    const int nl = a.bl - a.blo - 1, R = a.NP + 1;
    const long long total = (long long)a.rows * R * a.Ts;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int lp = (int)(i % a.Ts);
        const long long r = i / a.Ts;
        const int q = (int)(r % R), x = (int)(r / R);
        double v = 0.0;
        if (lp < nl && x < a.bl)
            v = q < a.NP ? a.G[((size_t)lp * a.NP + q) * a.Gs + x] : a.Bcoef[(size_t)(a.blo + 1 + lp) * a.Bp + x];
        a.out[i] = v;
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

// Stockham passes with the data of each pass in registers.  A CTA of T
// threads holds E = V*T complex values (V per thread): E/M transforms of size
// M (a power of two).  In a pass of radix R (R <= V) each thread owns V/R
// butterflies; butterfly (t,u) reads positions r*M + j + s*(M/R) and, after
// twiddles exp(SIGN 2 pi i (j mod Ns) s/(Ns R)) and a radix-R DFT, writes
// r*M + (j/Ns)*Ns*R + j%Ns + s*Ns.  The last pass (Ns = M/R) therefore writes
// exactly the positions the first pass of the same radix reads, so a forward
// FFT followed by an inverse FFT whose radices run in reverse order keeps the
// data in registers across the boundary.
template <int V, int R>
__device__ __forceinline__ int in_pos(int t, int u, int s, int lgM)
{
    constexpr int NB = V / R, LR = (R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : 4);
    const int b = t * NB + u, lper = lgM - LR, r = b >> lper, j = b & ((1 << lper) - 1);
    return (r << lgM) + j + (s << lper);
}

template <int V, int R, int SIGN>
__device__ __forceinline__ void bfly(double2 (&v)[V], int t, int lgM, int lNs, const double2 *twh,
                                     const double2 *twl)
{
    constexpr int NB = V / R, LR = (R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : 4);
#pragma unroll
    for (int u = 0; u < NB; u++) {
        if (lNs > 0) {
            const int b = t * NB + u, j = b & ((1 << (lgM - LR)) - 1), k = j & ((1 << lNs) - 1);
            const int step = k << (lgM - lNs - LR);
#pragma unroll
            for (int s = 1; s < R; s++) {
                double2 w = twid(twh, twl, step * s);
                if (SIGN > 0) w = cconj(w);
                v[u * R + s] = cmul(v[u * R + s], w);
            }
        }
        Dft<R, SIGN>::run(&v[u * R]);
    }
}

template <int V, int R>
__device__ __forceinline__ void store_pass(const double2 (&v)[V], double2 *buf, int t, int lgM, int lNs)
{
    constexpr int NB = V / R, LR = (R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : 4);
#pragma unroll
    for (int u = 0; u < NB; u++) {
        const int b = t * NB + u, lper = lgM - LR, r = b >> lper, j = b & ((1 << lper) - 1);
        const int idx = (r << lgM) + ((j >> lNs) << (lNs + LR)) + (j & ((1 << lNs) - 1));
#pragma unroll
        for (int s = 0; s < R; s++) buf[padix(idx + (s << lNs))] = v[u * R + s];
    }
}

template <int V, int R>
__device__ __forceinline__ void load_pass(double2 (&v)[V], const double2 *buf, int t, int lgM)
{
    constexpr int NB = V / R;
#pragma unroll
    for (int u = 0; u < NB; u++)
#pragma unroll
        for (int s = 0; s < R; s++) v[u * R + s] = buf[padix(in_pos<V, R>(t, u, s, lgM))];
}

// Radix plans for M = 2^k: forward [V,...,V,2^(k mod log2 V)], inverse in
// reverse order.  The radix of pass p is computed, not stored, so that no
// plan array is indexed dynamically.
struct RadixPlan {
    int np, nv, rem;
    bool rev;
    __device__ __forceinline__ int r(int p) const
    {
        if (rev) return (rem && p == 0) ? (1 << rem) : nv_radix;
        return (p < nv) ? nv_radix : (1 << rem);
    }
    int nv_radix;
};
template <int V>
__device__ __forceinline__ RadixPlan radix_plan(int lgM, bool reversed)
{
    constexpr int LV = (V == 8 ? 3 : 4);
    RadixPlan p;
    p.nv = lgM / LV;
    p.rem = lgM % LV;
    p.np = p.nv + (p.rem ? 1 : 0);
    p.rev = reversed;
    p.nv_radix = V;
    return p;
}

template <int V, int SIGN>
__device__ __forceinline__ void bfly_any(double2 (&v)[V], int R, int t, int lgM, int lNs, const double2 *twh,
                                         const double2 *twl)
{
    if (V == 16 && R == 16) bfly<V, (V >= 16 ? 16 : 2), SIGN>(v, t, lgM, lNs, twh, twl);
    else if (R == 8) bfly<V, 8, SIGN>(v, t, lgM, lNs, twh, twl);
    else if (R == 4) bfly<V, 4, SIGN>(v, t, lgM, lNs, twh, twl);
    else bfly<V, 2, SIGN>(v, t, lgM, lNs, twh, twl);
}
template <int V>
__device__ __forceinline__ void store_any(const double2 (&v)[V], int R, double2 *buf, int t, int lgM, int lNs)
{
    if (V == 16 && R == 16) store_pass<V, (V >= 16 ? 16 : 2)>(v, buf, t, lgM, lNs);
    else if (R == 8) store_pass<V, 8>(v, buf, t, lgM, lNs);
    else if (R == 4) store_pass<V, 4>(v, buf, t, lgM, lNs);
    else store_pass<V, 2>(v, buf, t, lgM, lNs);
}
template <int V>
__device__ __forceinline__ void load_any(double2 (&v)[V], int R, const double2 *buf, int t, int lgM)
{
    if (V == 16 && R == 16) load_pass<V, (V >= 16 ? 16 : 2)>(v, buf, t, lgM);
    else if (R == 8) load_pass<V, 8>(v, buf, t, lgM);
    else if (R == 4) load_pass<V, 4>(v, buf, t, lgM);
    else load_pass<V, 2>(v, buf, t, lgM);
}

template <int V, int SIGN>
__device__ __forceinline__ void fft_run(double2 (&v)[V], double2 *buf, int t, int lgM, const RadixPlan &P,
                                        const double2 *twh, const double2 *twl)
{
    int lNs = 0;
    for (int p = 0; p < P.np; p++) {
        const int R = P.r(p), LR = 31 - __clz(R);
        bfly_any<V, SIGN>(v, R, t, lgM, lNs, twh, twl);
        if (p + 1 < P.np) {
            store_any<V>(v, R, buf, t, lgM, lNs);
            __syncthreads();
            load_any<V>(v, P.r(p + 1), buf, t, lgM);
            __syncthreads();
        }
        lNs += LR;
    }
}

// Position (within the CTA buffer) of value i = u*R + s a thread holds for a
// pass of radix R.
template <int V>
__device__ __forceinline__ int pos_of(int i, int R, int t, int lgM)
{
    const int LR = 31 - __clz(R), u = i >> LR, s = i & (R - 1);
    const int b = t * (V / R) + u, lper = lgM - LR, r = b >> lper, j = b & ((1 << lper) - 1);
    return (r << lgM) + j + (s << lper);
}

// 32-byte accesses of the alpha stages (the two b columns of a b pair at
// one (g, m)): one 256-bit access instead of two 128-bit ones halves the
// L1 wavefronts of these row-strided loads and stores.  The streamed input
// is not kept in L1, which holds the chirp tables.
__device__ __forceinline__ void ld_pair(const double2 *p, double2 &a, double2 &b)
{
    asm("ld.global.nc.L1::no_allocate.v4.f64 {%0, %1, %2, %3}, [%4];"
        : "=d"(a.x), "=d"(a.y), "=d"(b.x), "=d"(b.y)
        : "l"(p));
}
__device__ __forceinline__ void st_pair(double2 *p, double2 a, double2 b)
{
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(a.x), "d"(a.y), "d"(b.x), "d"(b.y)
                 : "memory");
}

// Filter spectrum entry k of a Bluestein transform.  The alpha stages' filter
// h(d) = conj(chirp(d)) is even in d (no offsets), so its spectrum is even:
// Hf[k] = Hf[M - k]; reading only k <= M/2 halves the table's cache
// footprint (32 KB instead of 64 KB at M = 4096).
template <int MODE>
__device__ __forceinline__ double2 hf_at(const double2 *Hf, int k, int M)
{
    if (MODE == CZT_ANA_ALPHA || MODE == CZT_SYN_ALPHA) return Hf[k <= (M >> 1) ? k : M - k];
    return Hf[k];
}

// ---- beta transforms as FFTs of length L = 2 bl (Makhoul's algorithm) ----
// Analysis (s2dw_core_mod.f90:708-743), one row X(p), p < bl:
//   cos rows (m+N-1 even): Y(b) = sum_p c_p X(p) cos(p beta_b), c_0 = 1, c_p = 2,
//   sin rows (m+N-1 odd):  Y(b) = X(0) + sum_{p>=1} 2i X(p) sin(p beta_b),
// beta_b = pi (2b+1)/(2L), b < L.  The cos sum is a DCT-III of length L:
//   V_0 = X(0), V_k = e_k X(k) (0 < k < bl), V_bl = 0, V_k = conj(e_{L-k}) X(L-k) (k > bl),
//   v = sum_k V_k e^{+2 pi i k n/L},  Y(2n) = v_n, Y(2n+1) = v_{L-1-n}  (n < bl),
// e_k = exp(i pi k/(2L)) (the czt.pre table).  The sin sum is the same DCT-III
// of the reversed input times i(-1)^b, which moves factors -i (k < bl) and +i
// (k > bl) onto V and i, -i onto the two output halves; its V_0 is 0 and the
// reference's m' = 0 term X(0) (eta = 1) is added to every output.
// Synthesis (:1157-1198), one row u_b, b < L, folded over +-m':
//   cos rows (m+n even): V'(0) = sum_b u_b, V'(m') = 2 sum_b u_b cos(m' beta_b),
//   sin rows (m+n odd):  V'(m') = -2i sum_b u_b sin(m' beta_b),
// a DCT-II of length L: permute v_n = u_{2n}, v_{L-1-n} = u_{2n+1} (n < bl),
// V = sum_n v_n e^{-2 pi i k n/L}, V'(m') = conj(e_m') V_m' +- e_m' V_{L-m'}
// (+ cos, - sin; the sin rows' input carries (-1)^b).  A sin row's V'(0)
// multiplies d^l_{0m}(pi/2) d^l_{0n}(pi/2), which is zero for every l when m+n
// is odd, so it is stored as 0.

// Position b of the beta grid whose value sits at FFT index k in the
// DCT-II / DCT-III reordering (k < bl: b = 2k; k >= bl: b = 2L-1-2k).
__device__ __forceinline__ int beta_src(int k, int bl) { return k < bl ? 2 * k : 4 * bl - 1 - 2 * k; }

// DCT-III input V_k of the analysis beta transform of row X (bl values).
__device__ __forceinline__ double2 ana_beta_in(const double2 *X, int k, int bl, bool sn, const double2 *e)
{
    if (k == 0) return sn ? make_double2(0.0, 0.0) : X[0];
    if (k < bl) {
        const double2 x = cmul(X[k], e[k]);
        return sn ? make_double2(x.y, -x.x) : x;  // -i x
    }
    if (k == bl) return make_double2(0.0, 0.0);
    const int p = 2 * bl - k;
    const double2 x = cmul(X[p], cconj(e[p]));
    return sn ? make_double2(-x.y, x.x) : x;  // i x
}

// Output of the analysis beta transform held at FFT index j: its b, and the
// value (the sin rows' factor i or -i and the m' = 0 term x0 applied).
__device__ __forceinline__ double2 ana_beta_out(double2 y, int j, int bl, bool sn, double2 x0, int *b)
{
    if (j < bl) {
        *b = 2 * j;
        if (sn) y = make_double2(-y.y + x0.x, y.x + x0.y);  // i y + x0
    } else {
        *b = 4 * bl - 1 - 2 * j;
        if (sn) y = make_double2(y.y + x0.x, -y.x + x0.y);  // -i y + x0
    }
    return y;
}

// Folded synthesis beta output V'(m') from the FFT values at m' and L-m'.
__device__ __forceinline__ double2 syn_beta_out(double2 vk, double2 vlk, int mpv, bool sn, const double2 *e)
{
    if (mpv == 0) return sn ? make_double2(0.0, 0.0) : vk;
    const double2 y = cmul(vk, cconj(e[mpv])), z = cmul(vlk, e[mpv]);
    return sn ? csub(y, z) : cadd(y, z);
}

// Input element k of transform `row` of a MODE transform (pre-chirp or
// pre-twiddle applied); zero outside the transform's input range.
template <int MODE>
__device__ __forceinline__ double2 fft_load(const CztArgs &a, int row, int k, const double2 *ph)
{
    const int bl = a.bl, n = 2 * bl - 1, N = a.N;
    const double2 zero = make_double2(0.0, 0.0);
    if (MODE == CZT_ANA_ALPHA) {  // row = (g, b pair); Hermitian completion in m
        if (k >= n) return zero;
        const int g = row / bl, bp = row % bl;
        const bool lo = k < bl;
        const double2 *p = a.in_c + ((size_t)g * bl + (lo ? k : n - k)) * (2 * bl) + 2 * bp;
        double2 x1, x2;
        ld_pair(p, x1, x2);
        const double2 pr = a.czt.pre[k];
        if (!lo) { x1 = cconj(x1); x2 = cconj(x2); }
        if (k == 0) { x1.y = 0.0; x2.y = 0.0; }
        return cmul(make_double2(x1.x - x2.y, x1.y + x2.x), pr);
    } else if (MODE == CZT_SYN_ALPHA) {  // row = (g, b pair); z = w(:,b1) + i w(:,b2)
        if (k >= n) return zero;
        const int g = row / bl, bp = row % bl;
        const double *p = a.in_r + (size_t)k + (size_t)n * (2 * bp + (size_t)2 * bl * g);
        return cmul(make_double2(p[0], p[n]), a.czt.pre[k]);
    } else if (MODE == CZT_ANA_BETA) {  // row = (g, m); k <-> m' = k-(bl-1)
        if (k >= a.czt.spec.K) return zero;
        const int g = row / bl, m = row % bl, mpv = k - (bl - 1), ab = mpv < 0 ? -mpv : mpv;
        double2 x = a.in_c[((size_t)g * bl + m) * bl + ab];
        if (((m + N - 1) & 1) && mpv < 0) x = make_double2(-x.x, -x.y);
        return cmul(x, a.czt.pre[k]);
    } else if (MODE == FFT_ANA_BETA) {  // row = (g, m); DCT-III input V_k, k < L = 2bl
        const int g = row / bl, m = row % bl;
        return ana_beta_in(a.in_c + ((size_t)g * bl + m) * bl, k, bl, (m + N - 1) & 1, a.czt.pre);
    } else if (MODE == FFT_SYN_BETA) {  // row = (q, m); DCT-II input: u at b = beta_src(k), gamma DFT on the fly
        const int q = row / bl, m = row % bl, b = beta_src(k, bl);
        double2 u = zero;
        for (int g = 0; g < N; g++) u = cadd(u, cmul(a.in_c[((size_t)g * bl + m) * (2 * bl) + b], ph[q * N + g]));
        u = cscale(u, a.wq[b]);
        return (((m + a.nq[q]) & 1) && (b & 1)) ? make_double2(-u.x, -u.y) : u;
    } else {  // CZT_SYN_BETA: row = (q, m); k = b; gamma DFT on the fly
        if (k >= 2 * bl) return zero;
        const int q = row / bl, m = row % bl;
        double2 u = zero;
        for (int g = 0; g < N; g++) u = cadd(u, cmul(a.in_c[((size_t)g * bl + m) * (2 * bl) + k], ph[q * N + g]));
        u = cscale(u, a.wq[k]);
        return cmul(u, a.czt.pre[k]);
    }
}

template <int V, int THREADS, int MODE>
__global__ void __launch_bounds__(THREADS, (V * THREADS <= 4096 ? 2 : 1)) fft_kernel(CztArgs a)
{
    extern __shared__ double2 smem[];
    constexpr int E = V * THREADS;
    constexpr bool CHIRP = (MODE != FFT_ANA_BETA && MODE != FFT_SYN_BETA);
    constexpr bool SYNB = (MODE == CZT_SYN_BETA || MODE == FFT_SYN_BETA);
    const int M = a.czt.M, lgM = 31 - __clz(M), R = E / M;
    double2 *buf = smem;
    double2 *twh = smem + padix(E) + 1;
    const int nhi = (M + 63) / 64;
    double2 *twl = twh + nhi;
    double2 *ph = twl + 64;  // [q][g] exp(-i pi n_q g / N) for the synthesis beta modes
    const int t = threadIdx.x;
    const int bl = a.bl, n = 2 * bl - 1, N = a.N, Bout = a.czt.spec.Bout;
    const int row0 = blockIdx.x * R;

    for (int i = t; i < nhi; i += THREADS) twh[i] = a.tw.hi[i];
    for (int i = t; i < 64; i += THREADS) twl[i] = a.tw.lo[i];
    if (SYNB)
        for (int i = t; i < a.NP * N; i += THREADS) {
            const int q = i / N, g = i % N;
            double sn, cs;
            sincospi(-(double)(a.nq[q] * g) / (double)N, &sn, &cs);
            ph[i] = make_double2(cs, sn);
        }
    __syncthreads();

    const RadixPlan Pf = radix_plan<V>(lgM, false), Pi = radix_plan<V>(lgM, true);
    const int R0 = (MODE == FFT_ANA_BETA) ? Pi.r(0) : Pf.r(0);

    double2 v[V];
    if (MODE == FFT_SYN_BETA) {
        // the gamma DFT one sample (row of V) at a time, so that a thread's V
        // loads of one sample are in flight together (as fft_load, reordered)
        int src[V];
#pragma unroll
        for (int i = 0; i < V; i++) {
            const int pos = pos_of<V>(i, R0, t, lgM), row = row0 + (pos >> lgM);
            src[i] = row < a.rows ? (row % bl) * (2 * bl) + beta_src(pos & (M - 1), bl) : -1;
            v[i] = make_double2(0.0, 0.0);
        }
        for (int gg = 0; gg < N; gg++) {
            const double2 *Vg = a.in_c + (size_t)gg * bl * (2 * bl);
#pragma unroll
            for (int i = 0; i < V; i++) {
                if (src[i] < 0) continue;
                const int pos = pos_of<V>(i, R0, t, lgM), q = (row0 + (pos >> lgM)) / bl;
                v[i] = cadd(v[i], cmul(Vg[src[i]], ph[q * N + gg]));
            }
        }
#pragma unroll
        for (int i = 0; i < V; i++) {
            if (src[i] < 0) continue;
            const int pos = pos_of<V>(i, R0, t, lgM), row = row0 + (pos >> lgM), q = row / bl, m = row % bl;
            const int b = beta_src(pos & (M - 1), bl);
            const double2 u = cscale(v[i], a.wq[b]);
            v[i] = (((m + a.nq[q]) & 1) && (b & 1)) ? make_double2(-u.x, -u.y) : u;
        }
    } else {
#pragma unroll
        for (int i = 0; i < V; i++) {
            const int pos = pos_of<V>(i, R0, t, lgM), r = pos >> lgM, k = pos & (M - 1), row = row0 + r;
            v[i] = (row < a.rows) ? fft_load<MODE>(a, row, k, ph) : make_double2(0.0, 0.0);
        }
    }

    int RL;  // radix of the last pass run
    if (MODE == FFT_ANA_BETA) {
        fft_run<V, +1>(v, buf, t, lgM, Pi, twh, twl);
        RL = Pi.r(Pi.np - 1);
    } else if (MODE == FFT_SYN_BETA) {
        fft_run<V, -1>(v, buf, t, lgM, Pf, twh, twl);
        RL = Pf.r(Pf.np - 1);
    } else {
        fft_run<V, -1>(v, buf, t, lgM, Pf, twh, twl);
        const int RF = Pf.r(Pf.np - 1);
#pragma unroll
        for (int i = 0; i < V; i++) v[i] = cmul(v[i], hf_at<MODE>(a.czt.Hf, pos_of<V>(i, RF, t, lgM) & (M - 1), M));
        fft_run<V, +1>(v, buf, t, lgM, Pi, twh, twl);
        RL = Pi.r(Pi.np - 1);
    }

    // ---- store
    if (MODE == CZT_ANA_BETA || MODE == FFT_ANA_BETA || MODE == CZT_ANA_ALPHA) {
#pragma unroll
        for (int i = 0; i < V; i++) {
            const int pos = pos_of<V>(i, RL, t, lgM), r = pos >> lgM, b = pos & (M - 1), row = row0 + r;
            if (row >= a.rows || b >= Bout) continue;
            if (MODE == FFT_ANA_BETA) {
                const int g = row / bl, m = row % bl;
                const bool sn = (m + N - 1) & 1;
                const double2 *X = a.in_c + ((size_t)g * bl + m) * bl;
                int bo;
                const double2 y = ana_beta_out(v[i], b, bl, sn, sn ? X[0] : make_double2(0.0, 0.0), &bo);
                a.out_c[((size_t)g * bl + m) * (2 * bl) + bo] = y;
                continue;
            }
            const double2 y = CHIRP ? cmul(v[i], a.czt.post[b]) : v[i];
            if (MODE == CZT_ANA_ALPHA) {
                const int g = row / bl, bp = row % bl;
                double *p = a.out_r + (size_t)b + (size_t)n * (2 * bp + (size_t)2 * bl * g);
                p[0] = y.x;
                p[n] = y.y;
            } else {
                const int g = row / bl, m = row % bl;
                a.out_c[((size_t)g * bl + m) * (2 * bl) + b] = y;
            }
        }
        return;
    }
    // pair stores go through shared memory
    __syncthreads();
#pragma unroll
    for (int i = 0; i < V; i++) buf[padix(pos_of<V>(i, RL, t, lgM))] = v[i];
    __syncthreads();
    if (MODE == CZT_SYN_ALPHA) {
        for (int i = t; i < R * bl; i += THREADS) {
            const int r = i / bl, m = i % bl, row = row0 + r;
            if (row >= a.rows) continue;
            const int g = row / bl, bp = row % bl;
            const int mc = (m == 0) ? 0 : n - m;
            const double2 Z = cmul(buf[padix((r << lgM) + m)], a.czt.post[m]);
            const double2 Zc = cconj(cmul(buf[padix((r << lgM) + mc)], a.czt.post[mc]));
            const double2 sm = cadd(Z, Zc), d = csub(Z, Zc);
            const double hh = 0.5 * a.scale;
            st_pair(a.out_c + ((size_t)g * bl + m) * (2 * bl) + 2 * bp, make_double2(sm.x * hh, sm.y * hh),
                    make_double2(d.y * hh, -d.x * hh));
        }
        return;
    }
    // synthesis beta: V2(m') for m' in (-bl, bl), folded to m' >= 0
    for (int i = t; i < R * bl; i += THREADS) {
        const int r = i / bl, mpv = i % bl, row = row0 + r;
        if (row >= a.rows) continue;
        const int q = row / bl, m = row % bl;
        double2 y, z;
        if (MODE == CZT_SYN_BETA) {
            const int t0 = bl - 1 + mpv, t1 = bl - 1 - mpv;
            y = cmul(buf[padix((r << lgM) + t0)], a.czt.post[t0]);
            z = cmul(buf[padix((r << lgM) + t1)], a.czt.post[t1]);
            if (mpv > 0) {
                if ((m + a.nq[q]) & 1) z = make_double2(-z.x, -z.y);
                y = cadd(y, z);
            }
        } else {
            y = syn_beta_out(buf[padix((r << lgM) + mpv)], buf[padix((r << lgM) + ((M - mpv) & (M - 1)))], mpv,
                             (m + a.nq[q]) & 1, a.czt.pre);
        }
        a.out_c[((size_t)q * bl + m) * a.out_stride + mpv] = y;
    }
}

// ===========================================================================
// Large transforms (M = 4096, 8192): one transform per CTA, compile-time size
//
// Radix-16 Stockham passes with 16 values per thread (THREADS = M/16), the
// shape with the fewest shared-memory exchanges.  The twiddles of a pass are
// the powers w^s (s = 1..15) of one root w = W_M^step: w from the two-level
// table, w^2..w^15 by products (w^8 and w^4 squarings, then products), which
// keeps shared-memory traffic to the data exchanges.  The row (g, m) or
// (g, b pair) comes from the 2-D grid, so no integer division is needed.
// ===========================================================================
template <int SIGN>
__device__ __forceinline__ void twiddle_powers16(double2 (&v)[16], double2 w)
{
    if (SIGN > 0) w = cconj(w);
    const double2 w2 = cmul(w, w), w4 = cmul(w2, w2), w8 = cmul(w4, w4);
    const double2 w3 = cmul(w2, w), w5 = cmul(w4, w), w6 = cmul(w4, w2), w7 = cmul(w4, w3);
    v[1] = cmul(v[1], w);
    v[2] = cmul(v[2], w2);
    v[3] = cmul(v[3], w3);
    v[4] = cmul(v[4], w4);
    v[5] = cmul(v[5], w5);
    v[6] = cmul(v[6], w6);
    v[7] = cmul(v[7], w7);
    v[8] = cmul(v[8], w8);
    v[9] = cmul(v[9], cmul(w8, w));
    v[10] = cmul(v[10], cmul(w8, w2));
    v[11] = cmul(v[11], cmul(w8, w3));
    v[12] = cmul(v[12], cmul(w8, w4));
    v[13] = cmul(v[13], cmul(w8, w5));
    v[14] = cmul(v[14], cmul(w8, w6));
    v[15] = cmul(v[15], cmul(w8, w7));
}

// One radix-16 pass (16 values per thread, thread t = butterfly j).
template <int LGM, int LNS, int SIGN>
__device__ __forceinline__ void pass16(double2 (&v)[16], int t, const double2 *twh, const double2 *twl)
{
    if (LNS > 0) {
        const int k = t & ((1 << LNS) - 1);
        twiddle_powers16<SIGN>(v, twid(twh, twl, k << (LGM - LNS - 4)));
    }
    Dft<16, SIGN>::run(v);
}

// Radix-2 pass for LGM = 13 (the remainder of 13 = 4+4+4+1), 8 butterflies per thread.
template <int LGM, int LNS, int SIGN>
__device__ __forceinline__ void pass2x8(double2 (&v)[16], int t, const double2 *twh, const double2 *twl)
{
#pragma unroll
    for (int u = 0; u < 8; u++) {
        if (LNS > 0) {
            const int j = (t * 8 + u) & ((1 << (LGM - 1)) - 1), k = j & ((1 << LNS) - 1);
            double2 w = twid(twh, twl, k << (LGM - LNS - 1));
            if (SIGN > 0) w = cconj(w);
            v[2 * u + 1] = cmul(v[2 * u + 1], w);
        }
        const double2 a = v[2 * u], b = v[2 * u + 1];
        v[2 * u] = cadd(a, b);
        v[2 * u + 1] = csub(a, b);
    }
}

// Radix-8 pass for LGM = 11 (the remainder of 11 = 4+4+3), 2 butterflies per thread.
template <int LGM, int LNS, int SIGN>
__device__ __forceinline__ void pass8x2(double2 (&v)[16], int t, const double2 *twh, const double2 *twl)
{
#pragma unroll
    for (int u = 0; u < 2; u++) {
        if (LNS > 0) {
            const int j = (t * 2 + u) & ((1 << (LGM - 3)) - 1), k = j & ((1 << LNS) - 1);
            double2 w = twid(twh, twl, k << (LGM - LNS - 3));
            if (SIGN > 0) w = cconj(w);
            const double2 w2 = cmul(w, w), w3 = cmul(w2, w), w4 = cmul(w2, w2);
            v[8 * u + 1] = cmul(v[8 * u + 1], w);
            v[8 * u + 2] = cmul(v[8 * u + 2], w2);
            v[8 * u + 3] = cmul(v[8 * u + 3], w3);
            v[8 * u + 4] = cmul(v[8 * u + 4], w4);
            v[8 * u + 5] = cmul(v[8 * u + 5], cmul(w4, w));
            v[8 * u + 6] = cmul(v[8 * u + 6], cmul(w4, w2));
            v[8 * u + 7] = cmul(v[8 * u + 7], cmul(w4, w3));
        }
        Dft<8, SIGN>::run(&v[8 * u]);
    }
}

// Radix of the first pass of the forward (SIGN < 0) or inverse (SIGN > 0)
// transform of size 2^LGM, and of its last pass.
template <int LGM, int SIGN>
__host__ __device__ constexpr int first_radix()
{
    return SIGN < 0 ? 16 : (LGM == 13 ? 2 : LGM == 11 ? 8 : 16);
}
template <int LGM, int SIGN>
__host__ __device__ constexpr int last_radix()
{
    return SIGN > 0 ? 16 : (LGM == 13 ? 2 : LGM == 11 ? 8 : 16);
}

// Shared-memory exchange after a pass of radix R at LNS into the input
// positions of the next pass of radix RN (values per thread: 16).
template <int LGM, int R, int LNS, int RN>
__device__ __forceinline__ void exchange(double2 (&v)[16], double2 *buf, int t)
{
    constexpr int NB = 16 / R, LR = (R == 16 ? 4 : R == 8 ? 3 : 1), NBN = 16 / RN,
                  LRN = (RN == 16 ? 4 : RN == 8 ? 3 : 1);
#pragma unroll
    for (int u = 0; u < NB; u++) {
        const int j = t * NB + u;
        const int idx = ((j >> LNS) << (LNS + LR)) + (j & ((1 << LNS) - 1));
#pragma unroll
        for (int s = 0; s < R; s++) buf[padix(idx + (s << LNS))] = v[u * R + s];
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < NBN; u++) {
        const int j = t * NBN + u;
#pragma unroll
        for (int s = 0; s < RN; s++) v[u * RN + s] = buf[padix(j + (s << (LGM - LRN)))];
    }
    __syncthreads();
}

// Forward (SIGN=-1, radices 16,16,16[,2]) or inverse (SIGN=+1, [2,]16,16,16)
// FFT of the values in registers; input positions of the first pass, output
// positions of the last pass.
template <int LGM, int SIGN>
__device__ __forceinline__ void fft_large(double2 (&v)[16], double2 *buf, int t, const double2 *twh,
                                          const double2 *twl)
{
    if (LGM == 11 && SIGN < 0) {  // forward: 16,16,8
        pass16<11, 0, SIGN>(v, t, twh, twl);
        exchange<11, 16, 0, 16>(v, buf, t);
        pass16<11, 4, SIGN>(v, t, twh, twl);
        exchange<11, 16, 4, 8>(v, buf, t);
        pass8x2<11, 8, SIGN>(v, t, twh, twl);
    } else if (LGM == 11) {  // inverse: 8,16,16
        pass8x2<11, 0, SIGN>(v, t, twh, twl);
        exchange<11, 8, 0, 16>(v, buf, t);
        pass16<11, 3, SIGN>(v, t, twh, twl);
        exchange<11, 16, 3, 16>(v, buf, t);
        pass16<11, 7, SIGN>(v, t, twh, twl);
    } else if (LGM == 12) {
        pass16<12, 0, SIGN>(v, t, twh, twl);
        exchange<12, 16, 0, 16>(v, buf, t);
        pass16<12, 4, SIGN>(v, t, twh, twl);
        exchange<12, 16, 4, 16>(v, buf, t);
        pass16<12, 8, SIGN>(v, t, twh, twl);
    } else if (SIGN < 0) {  // LGM == 13 forward: 16,16,16,2
        pass16<13, 0, SIGN>(v, t, twh, twl);
        exchange<13, 16, 0, 16>(v, buf, t);
        pass16<13, 4, SIGN>(v, t, twh, twl);
        exchange<13, 16, 4, 16>(v, buf, t);
        pass16<13, 8, SIGN>(v, t, twh, twl);
        exchange<13, 16, 8, 2>(v, buf, t);
        pass2x8<13, 12, SIGN>(v, t, twh, twl);
    } else {  // LGM == 13 inverse: 2,16,16,16
        pass2x8<13, 0, SIGN>(v, t, twh, twl);
        exchange<13, 2, 0, 16>(v, buf, t);
        pass16<13, 1, SIGN>(v, t, twh, twl);
        exchange<13, 16, 1, 16>(v, buf, t);
        pass16<13, 5, SIGN>(v, t, twh, twl);
        exchange<13, 16, 5, 16>(v, buf, t);
        pass16<13, 9, SIGN>(v, t, twh, twl);
    }
}

// Position in [0, M) of value i held by thread t at the input of a pass of
// radix R (R = 16: i = s; R = 2: i = 2u + s).
template <int LGM, int R>
__device__ __forceinline__ int lpos(int t, int i)
{
    if (R == 16) return t + (i << (LGM - 4));
    if (R == 8) return ((t * 2 + (i >> 3)) & ((1 << (LGM - 3)) - 1)) + ((i & 7) << (LGM - 3));
    const int u = i >> 1, s = i & 1;
    return ((t * 8 + u) & ((1 << (LGM - 1)) - 1)) + (s << (LGM - 1));
}

template <int MODE, int LGM>
__global__ void __launch_bounds__((1 << LGM) / 16, (LGM == 11 ? 4 : LGM == 12 ? 2 : 1)) fft_large_kernel(CztArgs a)
{
    constexpr int M = 1 << LGM, THREADS = M / 16;
    constexpr bool CHIRP = (MODE != FFT_ANA_BETA && MODE != FFT_SYN_BETA);
    constexpr bool SYNB = (MODE == CZT_SYN_BETA || MODE == FFT_SYN_BETA);
    // first-pass radix of the transform run first, last-pass radix of the last
    constexpr int R0 = MODE == FFT_ANA_BETA ? first_radix<LGM, +1>() : first_radix<LGM, -1>();
    constexpr int RL = MODE == FFT_SYN_BETA ? last_radix<LGM, -1>() : last_radix<LGM, +1>();
    extern __shared__ double2 smem[];
    double2 *buf = smem;
    double2 *twh = smem + padix(M) + 1;
    double2 *twl = twh + M / 64;
    double2 *ph = twl + 64;
    const int t = threadIdx.x;
    const int bl = a.bl, n = 2 * bl - 1, N = a.N, Bout = a.czt.spec.Bout;
    // row = (g or q, m or b pair); the synthesis beta modes put q on the fast
    // grid axis so that the CTAs of one m, which read the same N rows of V,
    // run together and the repeated reads hit L2
    const int g = SYNB ? blockIdx.x : blockIdx.y, rr = SYNB ? blockIdx.y : blockIdx.x;
    const double2 zero = make_double2(0.0, 0.0);

    for (int i = t; i < M / 64; i += THREADS) twh[i] = a.tw.hi[i];
    for (int i = t; i < 64; i += THREADS) twl[i] = a.tw.lo[i];
    if (SYNB && t < N) {
        double sn, cs;
        sincospi(-(double)(a.nq[g] * t) / (double)N, &sn, &cs);
        ph[t] = make_double2(cs, sn);
    }
    __syncthreads();

    double2 v[16];
    if (MODE == FFT_SYN_BETA) {
        // gamma DFT of the row with coalesced loads (b contiguous across the
        // threads), then the DCT-II reordering through shared memory: the
        // value of b goes to FFT index b/2 (b even) or (4bl-1-b)/2 (b odd)
        const bool sn = (rr + a.nq[g]) & 1;
        // one gamma sample (row of V) at a time: its 16 loads per thread are
        // independent, so they are all in flight together
#pragma unroll
        for (int i = 0; i < 16; i++) v[i] = zero;
        for (int gg = 0; gg < N; gg++) {
            const double2 *row = a.in_c + ((size_t)gg * bl + rr) * (2 * bl);
            const double2 w = ph[gg];
#pragma unroll
            for (int i = 0; i < 16; i++) v[i] = cadd(v[i], cmul(row[t + i * THREADS], w));
        }
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const int b = t + i * THREADS;
            double2 u = cscale(v[i], a.wq[b]);
            if (sn && (b & 1)) u = make_double2(-u.x, -u.y);
            buf[padix((b & 1) ? (4 * bl - 1 - b) >> 1 : b >> 1)] = u;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 16; i++) v[i] = buf[padix(lpos<LGM, R0>(t, i))];
        __syncthreads();  // the exchanges of the FFT reuse buf
    }
#pragma unroll
    for (int i = 0; i < 16 && MODE != FFT_SYN_BETA; i++) {
        const int k = lpos<LGM, R0>(t, i);
        double2 x = zero;
        if (MODE == CZT_ANA_ALPHA) {  // (g, b pair rr); Hermitian completion in m
            if (k < n) {
                const bool lo = k < bl;
                const double2 *p = a.in_c + ((size_t)g * bl + (lo ? k : n - k)) * (2 * bl) + 2 * rr;
                double2 x1, x2;
                ld_pair(p, x1, x2);
                if (!lo) { x1 = cconj(x1); x2 = cconj(x2); }
                if (k == 0) { x1.y = 0.0; x2.y = 0.0; }
                x = cmul(make_double2(x1.x - x2.y, x1.y + x2.x), a.czt.pre[k]);
            }
        } else if (MODE == CZT_SYN_ALPHA) {  // (g, b pair rr)
            if (k < n) {
                const double *p = a.in_r + (size_t)k + (size_t)n * (2 * rr + (size_t)2 * bl * g);
                x = cmul(make_double2(p[0], p[n]), a.czt.pre[k]);
            }
        } else if (MODE == CZT_ANA_BETA) {  // (g, m = rr)
            if (k < a.czt.spec.K) {
                const int mpv = k - (bl - 1), ab = mpv < 0 ? -mpv : mpv;
                x = a.in_c[((size_t)g * bl + rr) * bl + ab];
                if (((rr + N - 1) & 1) && mpv < 0) x = make_double2(-x.x, -x.y);
                x = cmul(x, a.czt.pre[k]);
            }
        } else if (MODE == FFT_ANA_BETA) {  // (g, m = rr), DCT-III input
            x = ana_beta_in(a.in_c + ((size_t)g * bl + rr) * bl, k, bl, (rr + N - 1) & 1, a.czt.pre);
        } else {  // CZT_SYN_BETA, (q = g, m = rr), k = b
            if (k < 2 * bl) {
                double2 u = zero;
                for (int gg = 0; gg < N; gg++)
                    u = cadd(u, cmul(a.in_c[((size_t)gg * bl + rr) * (2 * bl) + k], ph[gg]));
                x = cmul(cscale(u, a.wq[k]), a.czt.pre[k]);
            }
        }
        v[i] = x;
    }

    if (MODE == FFT_ANA_BETA) {
        fft_large<LGM, +1>(v, buf, t, twh, twl);
    } else if (MODE == FFT_SYN_BETA) {
        fft_large<LGM, -1>(v, buf, t, twh, twl);
    } else {
        fft_large<LGM, -1>(v, buf, t, twh, twl);
        constexpr int RF = last_radix<LGM, -1>();
#pragma unroll
        for (int i = 0; i < 16; i++) v[i] = cmul(v[i], hf_at<MODE>(a.czt.Hf, lpos<LGM, RF>(t, i), M));
        fft_large<LGM, +1>(v, buf, t, twh, twl);
    }

    if (MODE == CZT_ANA_BETA || MODE == FFT_ANA_BETA || MODE == CZT_ANA_ALPHA) {
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const int b = lpos<LGM, RL>(t, i);
            if (b >= Bout) continue;
            if (MODE == FFT_ANA_BETA) {
                const bool sn = (rr + N - 1) & 1;
                const double2 *X = a.in_c + ((size_t)g * bl + rr) * bl;
                int bo;
                const double2 y = ana_beta_out(v[i], b, bl, sn, sn ? X[0] : zero, &bo);
                a.out_c[((size_t)g * bl + rr) * (2 * bl) + bo] = y;
                continue;
            }
            const double2 y = CHIRP ? cmul(v[i], a.czt.post[b]) : v[i];
            if (MODE == CZT_ANA_ALPHA) {
                double *p = a.out_r + (size_t)b + (size_t)n * (2 * rr + (size_t)2 * bl * g);
                p[0] = y.x;
                p[n] = y.y;
            } else {
                a.out_c[((size_t)g * bl + rr) * (2 * bl) + b] = y;
            }
        }
        return;
    }
    // pair stores through shared memory
#pragma unroll
    for (int i = 0; i < 16; i++) buf[padix(lpos<LGM, RL>(t, i))] = v[i];
    __syncthreads();
    if (MODE == CZT_SYN_ALPHA) {
        for (int m = t; m < bl; m += THREADS) {
            const int mc = (m == 0) ? 0 : n - m;
            const double2 Z = cmul(buf[padix(m)], a.czt.post[m]);
            const double2 Zc = cconj(cmul(buf[padix(mc)], a.czt.post[mc]));
            const double2 sm = cadd(Z, Zc), d = csub(Z, Zc);
            const double hh = 0.5 * a.scale;
            st_pair(a.out_c + ((size_t)g * bl + m) * (2 * bl) + 2 * rr, make_double2(sm.x * hh, sm.y * hh),
                    make_double2(d.y * hh, -d.x * hh));
        }
        return;
    }
    for (int mpv = t; mpv < bl; mpv += THREADS) {
        double2 y;
        if (MODE == CZT_SYN_BETA) {
            const int t0 = bl - 1 + mpv, t1 = bl - 1 - mpv;
            y = cmul(buf[padix(t0)], a.czt.post[t0]);
            double2 z = cmul(buf[padix(t1)], a.czt.post[t1]);
            if (mpv > 0) {
                if ((rr + a.nq[g]) & 1) z = make_double2(-z.x, -z.y);
                y = cadd(y, z);
            }
        } else {
            y = syn_beta_out(buf[padix(mpv)], buf[padix((M - mpv) & (M - 1))], mpv, (rr + a.nq[g]) & 1, a.czt.pre);
        }
        a.out_c[((size_t)g * bl + rr) * a.out_stride + mpv] = y;
    }
}

// ===========================================================================
// Stages with the input prefetched (M = 4096, 8192): synthesis alpha and
// analysis beta
//
// A persistent form of fft_large_kernel for the two modes whose input row is
// contiguous in HBM: each CTA loops over rows and copies the next row's input
// into shared memory with cp.async while the current row's transforms run,
// so the input's DRAM latency is hidden behind the FFT arithmetic instead of
// stalling every warp of the CTA at the start of each row.  The twiddle
// tables are loaded once per CTA.  Staged input per row:
//   CZT_SYN_ALPHA (row = (g, b pair)): the two real rows of the b pair,
//     2n contiguous doubles at a multiple of 2n doubles from in_r;
//   FFT_ANA_BETA (row = (g, m)): Tg(g, m, 0..bl-1), bl complex values.
// ===========================================================================
__device__ __forceinline__ void pf_cp16(void *smem, const void *gmem)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void pf_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void pf_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// 16-byte chunks of one row's staged input.
template <int MODE>
__host__ __device__ constexpr int pf_chunks(int bl)
{
    return MODE == CZT_SYN_ALPHA ? 2 * bl - 1 : bl;
}

// Issues the copies of row r's input into stg.
template <int MODE, int THREADS>
__device__ __forceinline__ void pf_prefetch(const CztArgs &a, int r, double2 *stg, int t)
{
    const int bl = a.bl, n = 2 * bl - 1, g = r / bl, rr = r - g * bl;
    const double2 *base;
    if (MODE == CZT_SYN_ALPHA)
        base = reinterpret_cast<const double2 *>(a.in_r + (size_t)n * (2 * rr + (size_t)2 * bl * g));
    else
        base = a.in_c + ((size_t)g * bl + rr) * bl;
    for (int i = t; i < pf_chunks<MODE>(bl); i += THREADS) pf_cp16(stg + i, base + i);
}

template <int MODE, int LGM>
__global__ void __launch_bounds__((1 << LGM) / 16, (LGM == 11 ? 4 : LGM == 12 ? 2 : 1)) fft_pf_kernel(CztArgs a)
{
    static_assert(MODE == CZT_SYN_ALPHA || MODE == FFT_ANA_BETA, "contiguous-input stages only");
    constexpr int M = 1 << LGM, THREADS = M / 16;
    // first-pass radix of the transform run first (as fft_large_kernel)
    constexpr int R0 = MODE == FFT_ANA_BETA ? first_radix<LGM, +1>() : first_radix<LGM, -1>();
    extern __shared__ double2 smem[];
    double2 *buf = smem;
    double2 *twh = smem + padix(M) + 1;
    double2 *twl = twh + M / 64;
    double2 *stg = twl + 64;
    const int t = threadIdx.x;
    const int bl = a.bl, n = 2 * bl - 1, rows = a.rows, N = a.N, Bout = a.czt.spec.Bout;
    const double2 zero = make_double2(0.0, 0.0);

    for (int i = t; i < M / 64; i += THREADS) twh[i] = a.tw.hi[i];
    for (int i = t; i < 64; i += THREADS) twl[i] = a.tw.lo[i];
    if ((int)blockIdx.x < rows) pf_prefetch<MODE, THREADS>(a, blockIdx.x, stg, t);
    pf_commit();

    for (int r = blockIdx.x; r < rows; r += gridDim.x) {
        const int g = r / bl, rr = r - g * bl;
        pf_wait_all();
        __syncthreads();  // row r staged; the previous row's reads of buf done
        double2 v[16];
        bool sn = false;     // FFT_ANA_BETA: sin row
        double2 x0 = zero;   // FFT_ANA_BETA: the row's X(0)
        if (MODE == CZT_SYN_ALPHA) {
            const double *sd = reinterpret_cast<const double *>(stg);
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const int k = lpos<LGM, R0>(t, i);
                v[i] = (k < n) ? cmul(make_double2(sd[k], sd[n + k]), a.czt.pre[k]) : zero;
            }
        } else {  // DCT-III input, as fft_large_kernel's FFT_ANA_BETA load
            sn = (rr + N - 1) & 1;
            x0 = stg[0];
#pragma unroll
            for (int i = 0; i < 16; i++) v[i] = ana_beta_in(stg, lpos<LGM, R0>(t, i), bl, sn, a.czt.pre);
        }
        __syncthreads();  // staging free: copy the next row while this one runs
        if (r + (int)gridDim.x < rows) pf_prefetch<MODE, THREADS>(a, r + gridDim.x, stg, t);
        pf_commit();

        if (MODE == CZT_SYN_ALPHA) {
            fft_large<LGM, -1>(v, buf, t, twh, twl);
            constexpr int RF = last_radix<LGM, -1>();
#pragma unroll
            for (int i = 0; i < 16; i++) v[i] = cmul(v[i], hf_at<MODE>(a.czt.Hf, lpos<LGM, RF>(t, i), M));
            fft_large<LGM, +1>(v, buf, t, twh, twl);
            // pair split through shared memory, as fft_large_kernel
#pragma unroll
            for (int i = 0; i < 16; i++) buf[padix(lpos<LGM, 16>(t, i))] = v[i];
            __syncthreads();
            for (int m = t; m < bl; m += THREADS) {
                const int mc = (m == 0) ? 0 : n - m;
                const double2 Z = cmul(buf[padix(m)], a.czt.post[m]);
                const double2 Zc = cconj(cmul(buf[padix(mc)], a.czt.post[mc]));
                const double2 sm = cadd(Z, Zc), d = csub(Z, Zc);
                const double hh = 0.5 * a.scale;
                st_pair(a.out_c + ((size_t)g * bl + m) * (2 * bl) + 2 * rr, make_double2(sm.x * hh, sm.y * hh),
                        make_double2(d.y * hh, -d.x * hh));
            }
        } else {
            fft_large<LGM, +1>(v, buf, t, twh, twl);
#pragma unroll
            for (int i = 0; i < 16; i++) {
                int b;
                const double2 y = ana_beta_out(v[i], lpos<LGM, 16>(t, i), bl, sn, x0, &b);
                a.out_c[((size_t)g * bl + rr) * (2 * bl) + b] = y;
            }
        }
    }
    pf_wait_all();
}

// ===========================================================================
// Prime-factor alpha stages at bl = 2048: n = 2bl-1 = 4095 = 5 * 7 * 9 * 13
//
// For the smooth odd length of the full-band scales at B = 2048 the alpha
// transforms (the c2r of s2dw_core_mod.f90:746-768 and the r2c of :1104-1130,
// two real rows packed into one complex transform as in the Bluestein
// engines) run as a Good-Thomas prime-factor DFT: the 4095 values of a row go
// into shared memory in the 4-D layout L = d1 + 5 d2 + 35 d3 + 315 d4 with
// input digits d_i = (n u_i) mod R_i, u_i = (4095/R_i)^-1 mod R_i = 4, 2, 2, 9;
// plain DFTs of length R_i = 5, 7, 9, 13 run along each dimension in place (no
// twiddles between them); output k sits at digits k mod R_i.  Each small DFT
// uses the symmetric pairs x_k +- x_{R-k}: (R-1)^2 real-by-complex products
// instead of R^2.  About 40 FP64 operations per point against ~240 for the
// 8192-point Bluestein convolution of the general engine.
// ===========================================================================
// Load phase of the prime-factor alpha kernels: the row pair (g, rr) of one
// transform of odd length N into shared memory, value m at X[pos(m)], with
// all of a thread's global loads in flight before the first shared store.
// Analysis: only the rows m < bl = (N+1)/2 are read; the Hermitian completion
// m >= bl is their conjugate (z(N - m) from the same two values).  Synthesis:
// the two real rows, z = w(:, b1) + i w(:, b2).
template <int MODE, int NT, int N, typename Pos>
__device__ __forceinline__ void pfa_load(const CztArgs &a, double2 *X, Pos pos)
{
    constexpr int BL = (N + 1) / 2;
    const int t = threadIdx.x, g = blockIdx.y, rr = blockIdx.x;
    if (MODE == CZT_ANA_ALPHA) {
        constexpr int PB = (BL + NT - 1) / NT;
        double2 x1[PB], x2[PB];
#pragma unroll
        for (int i = 0; i < PB; i++) {
            const int m = t + i * NT;
            if (m < BL) ld_pair(a.in_c + ((size_t)g * BL + m) * (2 * BL) + 2 * rr, x1[i], x2[i]);
        }
#pragma unroll
        for (int i = 0; i < PB; i++) {
            const int m = t + i * NT;
            if (m < BL) {
                if (m == 0) { x1[i].y = 0.0; x2[i].y = 0.0; }
                X[pos(m)] = make_double2(x1[i].x - x2[i].y, x1[i].y + x2[i].x);
                if (m > 0) X[pos(N - m)] = make_double2(x1[i].x + x2[i].y, x2[i].x - x1[i].y);
            }
        }
    } else {
        constexpr int PB = (N + NT - 1) / NT;
        const double *p = a.in_r + (size_t)N * (2 * rr + (size_t)2 * BL * g);
        double z0[PB], z1[PB];
#pragma unroll
        for (int i = 0; i < PB; i++) {
            const int m = t + i * NT;
            if (m < N) {
                z0[i] = p[m];
                z1[i] = p[N + m];
            }
        }
#pragma unroll
        for (int i = 0; i < PB; i++) {
            const int m = t + i * NT;
            if (m < N) X[pos(m)] = make_double2(z0[i], z1[i]);
        }
    }
}

constexpr int PFA_N = 4095, PFA_THREADS = 256;

// cos(2 pi j / R) and sin(2 pi j / R), j < R (local constant tables: with j
// known after unrolling they fold into immediates)
template <int R>
__device__ __forceinline__ void pfa_cs(int j, double &c, double &s);
template <>
__device__ __forceinline__ void pfa_cs<5>(int j, double &c, double &s)
{
    constexpr double C[5] = {1.0, 0.309016994374947424102, -0.809016994374947424102, -0.809016994374947424102, 0.309016994374947424102};
    constexpr double S[5] = {0.0, 0.951056516295153572116, 0.587785252292473129169, -0.587785252292473129169, -0.951056516295153572116};
    c = C[j];
    s = S[j];
}
template <>
__device__ __forceinline__ void pfa_cs<7>(int j, double &c, double &s)
{
    constexpr double C[7] = {1.0, 0.623489801858733530525, -0.222520933956314404289, -0.900968867902419126236, -0.900968867902419126236, -0.222520933956314404289, 0.623489801858733530525};
    constexpr double S[7] = {0.0, 0.781831482468029808708, 0.974927912181823607018, 0.433883739117558120476, -0.433883739117558120476, -0.974927912181823607018, -0.781831482468029808708};
    c = C[j];
    s = S[j];
}
template <>
__device__ __forceinline__ void pfa_cs<9>(int j, double &c, double &s)
{
    constexpr double C[9] = {1.0, 0.766044443118978035202, 0.173648177666930348852, -0.5, -0.939692620785908384054, -0.939692620785908384054, -0.5, 0.173648177666930348852, 0.766044443118978035202};
    constexpr double S[9] = {0.0, 0.642787609686539326323, 0.984807753012208059367, 0.866025403784438646764, 0.342020143325668733044, -0.342020143325668733044, -0.866025403784438646764, -0.984807753012208059367, -0.642787609686539326323};
    c = C[j];
    s = S[j];
}
template <>
__device__ __forceinline__ void pfa_cs<13>(int j, double &c, double &s)
{
    constexpr double C[13] = {1.0, 0.885456025653209895900, 0.568064746731155802512, 0.120536680255323053349, -0.354604887042535625970, -0.748510748171101098635, -0.970941817426052027157, -0.970941817426052027157, -0.748510748171101098635, -0.354604887042535625970, 0.120536680255323053349, 0.568064746731155802512, 0.885456025653209895900};
    constexpr double S[13] = {0.0, 0.464723172043768545656, 0.822983865893656394580, 0.992708874098053992801, 0.935016242685414823440, 0.663122658240795202377, 0.239315664287557767149, -0.239315664287557767149, -0.663122658240795202377, -0.935016242685414823440, -0.992708874098053992801, -0.822983865893656394580, -0.464723172043768545656};
    c = C[j];
    s = S[j];
}

// In-place DFT of length R (odd) with exp(SIGN 2 pi i k m / R):
// y_m = x_0 + sum_k (x_k + x_{R-k}) cos + SIGN i sum_k (x_k - x_{R-k}) sin.
template <int R, int SIGN>
__device__ __forceinline__ void pfa_dft(double2 (&x)[R])
{
    constexpr int H = (R - 1) / 2;
    double2 ap[H], am[H];
    double2 y0 = x[0];
#pragma unroll
    for (int k = 1; k <= H; k++) {
        ap[k - 1] = cadd(x[k], x[R - k]);
        am[k - 1] = csub(x[k], x[R - k]);
        y0 = cadd(y0, ap[k - 1]);
    }
    const double2 x0 = x[0];
    x[0] = y0;
#pragma unroll
    for (int m = 1; m <= H; m++) {
        double2 P = x0, Q = make_double2(0.0, 0.0);
#pragma unroll
        for (int k = 1; k <= H; k++) {
            double c, sn;
            pfa_cs<R>((k * m) % R, c, sn);
            P.x = fma(ap[k - 1].x, c, P.x);
            P.y = fma(ap[k - 1].y, c, P.y);
            Q.x = fma(am[k - 1].x, sn, Q.x);
            Q.y = fma(am[k - 1].y, sn, Q.y);
        }
        // SIGN i Q
        const double2 iq = SIGN > 0 ? make_double2(-Q.y, Q.x) : make_double2(Q.y, -Q.x);
        x[m] = cadd(P, iq);
        x[R - m] = csub(P, iq);
    }
}

// DFTs of length R along the dimension of stride S of the 4-D layout.
template <int R, int S, int SIGN>
__device__ __forceinline__ void pfa_stage(double2 *sm, int t)
{
    for (int d = t; d < PFA_N / R; d += PFA_THREADS) {
        const int base = (d % S) + (d / S) * (S * R);
        double2 x[R];
#pragma unroll
        for (int r = 0; r < R; r++) x[r] = sm[base + r * S];
        pfa_dft<R, SIGN>(x);
#pragma unroll
        for (int r = 0; r < R; r++) sm[base + r * S] = x[r];
    }
}

__device__ __forceinline__ int pfa_in_pos(int n)
{
    return (n * 4) % 5 + 5 * ((n * 2) % 7) + 35 * ((n * 2) % 9) + 315 * ((n * 9) % 13);
}
__device__ __forceinline__ int pfa_out_pos(int k) { return k % 5 + 5 * (k % 7) + 35 * (k % 9) + 315 * (k % 13); }

// One CTA per (g, b pair): the two real rows of the pair, as fft_large_kernel.
template <int MODE>
__global__ void __launch_bounds__(PFA_THREADS, 3) pfa_alpha_kernel(CztArgs a)
{
    static_assert(MODE == CZT_ANA_ALPHA || MODE == CZT_SYN_ALPHA, "alpha stages only");
    constexpr int SIGN = MODE == CZT_ANA_ALPHA ? +1 : -1;
    extern __shared__ double2 smem[];
    const int t = threadIdx.x;
    const int bl = a.bl, n = PFA_N;  // n = 2 bl - 1
    const int g = blockIdx.y, rr = blockIdx.x;
    pfa_load<MODE, PFA_THREADS, PFA_N>(a, smem, [](int m) { return pfa_in_pos(m); });
    __syncthreads();
    pfa_stage<5, 1, SIGN>(smem, t);
    __syncthreads();
    pfa_stage<7, 5, SIGN>(smem, t);
    __syncthreads();
    pfa_stage<9, 35, SIGN>(smem, t);
    __syncthreads();
    pfa_stage<13, 315, SIGN>(smem, t);
    __syncthreads();
    if (MODE == CZT_ANA_ALPHA) {
        for (int k = t; k < n; k += PFA_THREADS) {
            const double2 y = smem[pfa_out_pos(k)];
            double *p = a.out_r + (size_t)k + (size_t)n * (2 * rr + (size_t)2 * bl * g);
            p[0] = y.x;
            p[n] = y.y;
        }
    } else {  // even / odd split of the two real rows' spectra, m < bl
        const double hh = 0.5 * a.scale;
        for (int m = t; m < bl; m += PFA_THREADS) {
            const double2 Z = smem[pfa_out_pos(m)];
            const double2 Zc = cconj(smem[pfa_out_pos(m == 0 ? 0 : n - m)]);
            const double2 sm = cadd(Z, Zc), d = csub(Z, Zc);
            st_pair(a.out_c + ((size_t)g * bl + m) * (2 * bl) + 2 * rr, make_double2(sm.x * hh, sm.y * hh),
                    make_double2(d.y * hh, -d.x * hh));
        }
    }
}

template <>
__device__ __forceinline__ void pfa_cs<11>(int j, double &c, double &s)
{
    constexpr double C[11] = {
        1.00000000000000000000, 0.841253532831181168862, 0.415415013001886425529, -0.142314838273285140444,
        -0.654860733945285064057, -0.959492973614497389890, -0.959492973614497389890, -0.654860733945285064057,
        -0.142314838273285140444, 0.415415013001886425529, 0.841253532831181168862};
    constexpr double S[11] = {
        0.0, 0.540640817455597582108, 0.909631995354518371412, 0.989821441880932732376, 0.755749574354258283774,
        0.281732556841429697711, -0.281732556841429697711, -0.755749574354258283774, -0.989821441880932732376,
        -0.909631995354518371412, -0.540640817455597582108};
    c = C[j];
    s = S[j];
}
template <>
__device__ __forceinline__ void pfa_cs<23>(int j, double &c, double &s)
{
    constexpr double C[23] = {
        1.00000000000000000000, 0.962917287347799295015, 0.854419404546488552548, 0.682553143218654082875,
        0.460065037731152126042, 0.203456013052633789878, -0.0682424133646709759212, -0.334879612170986151958,
        -0.576680322114867141251, -0.775711290704419807041, -0.917211301505453017844, -0.990685946036330752342,
        -0.990685946036330752342, -0.917211301505453017844, -0.775711290704419807041, -0.576680322114867141251,
        -0.334879612170986151958, -0.0682424133646709759212, 0.203456013052633789878, 0.460065037731152126042,
        0.682553143218654082875, 0.854419404546488552548, 0.962917287347799295015};
    constexpr double S[23] = {
        0.0, 0.269796771157024271245, 0.519583950035433578133, 0.730835964278124101651, 0.887885218402375234984,
        0.979084087682322875633, 0.997668769190539198454, 0.942260922118820495618, 0.816969893010442016973,
        0.631087944326052789367, 0.398401089846241457998, 0.136166649096246590761, -0.136166649096246590761,
        -0.398401089846241457998, -0.631087944326052789367, -0.816969893010442016973, -0.942260922118820495618,
        -0.997668769190539198454, -0.979084087682322875633, -0.887885218402375234984, -0.730835964278124101651,
        -0.519583950035433578133, -0.269796771157024271245};
    c = C[j];
    s = S[j];
}

// In-place-input DFT of length R (odd), outputs written to out[base + m S]:
// the symmetric pairs overwrite x (x_k <- x_k + x_{R-k}, x_{R-k} <- x_k - x_{R-k}),
// which keeps the registers of a long DFT (R = 23) to about R complex values.
template <int R, int SIGN>
__device__ __forceinline__ void pfa_dft_out(double2 (&x)[R], double2 *out, int base, int S)
{
    constexpr int H = (R - 1) / 2;
    const double2 x0 = x[0];
    double2 y0 = x0;
#pragma unroll
    for (int k = 1; k <= H; k++) {
        const double2 p = cadd(x[k], x[R - k]), q = csub(x[k], x[R - k]);
        x[k] = p;
        x[R - k] = q;
        y0 = cadd(y0, p);
    }
    out[base] = y0;
#pragma unroll
    for (int m = 1; m <= H; m++) {
        double2 P = x0, Q = make_double2(0.0, 0.0);
#pragma unroll
        for (int k = 1; k <= H; k++) {
            double c, sn;
            pfa_cs<R>((k * m) % R, c, sn);
            P.x = fma(x[k].x, c, P.x);
            P.y = fma(x[k].y, c, P.y);
            Q.x = fma(x[R - k].x, sn, Q.x);
            Q.y = fma(x[R - k].y, sn, Q.y);
        }
        const double2 iq = SIGN > 0 ? make_double2(-Q.y, Q.x) : make_double2(Q.y, -Q.x);
        out[base + m * S] = cadd(P, iq);
        out[base + (R - m) * S] = csub(P, iq);
    }
}

// ---------------------------------------------------------------------------
// Prime-factor alpha stages at bl = 1024: n = 2047 = 23 * 89
//
// Good-Thomas over 23 x 89 as above (layout L = d1 + 23 d2, input digits
// (n 15) mod 23 and (n 31) mod 89, output digits k mod 23, k mod 89).  The
// length-89 DFTs run by Rader's algorithm: with the primitive root g = 3,
// y_{g^r} = x_0 + sum_q x_{g^-q} w_{r-q}, w_j = exp(SIGN 2 pi i g^j / 89), a cyclic
// convolution of length 88 done as a forward DFT of 88 = 8 x 11 (Good-Thomas
// again: radix-8 in registers, then length 11), a product with the DFT of w
// (g_rader_w, built once per device by rader_init_kernel), and the inverse
// DFT; y_0 = x_0 + the convolution input's sum.  About 60 FP64 operations per
// point against ~240 for the 4096-point Bluestein convolution.
// ---------------------------------------------------------------------------
constexpr int PFB_N = 2047;
constexpr int PFB_P = 25;              // pitch of d2 in the shared row
constexpr int PFB_XS = PFB_P * 89;     // shared row size
constexpr int PFB_SP = 103;            // pitch of a Rader column (positions i + 9 j, i < 8, j < 11)

// per position L = i + 8 j of the 88-layout (input digits (q 3) mod 8,
// (q 7) mod 11): the length-89 index g^-q whose value goes there, and g^q,
// where the convolution's output at L goes
__constant__ int c_rader_src[88] = {
    1, 77, 55, 52, 88, 12, 34, 37, 32, 61, 69, 62, 57, 28, 20, 27, 45, 83, 72, 26, 44, 6, 17, 63, 16, 75, 79, 31,
    73, 14, 10, 58, 67, 86, 36, 13, 22, 3, 53, 76, 8, 82, 84, 60, 81, 7, 5, 29, 78, 43, 18, 51, 11, 46, 71, 38, 4,
    41, 42, 30, 85, 48, 47, 59, 39, 66, 9, 70, 50, 23, 80, 19, 2, 65, 21, 15, 87, 24, 68, 74, 64, 33, 49, 35, 25,
    56, 40, 54};
__constant__ int c_rader_dst[88] = {
    1, 37, 34, 12, 88, 52, 55, 77, 64, 54, 40, 56, 25, 35, 49, 33, 2, 74, 68, 24, 87, 15, 21, 65, 39, 19, 80, 23,
    50, 70, 9, 66, 4, 59, 47, 48, 85, 30, 42, 41, 78, 38, 71, 46, 11, 51, 18, 43, 8, 29, 5, 7, 81, 60, 84, 82, 67,
    76, 53, 3, 22, 13, 36, 86, 16, 58, 10, 14, 73, 31, 79, 75, 45, 63, 17, 6, 44, 26, 72, 83, 32, 27, 20, 28, 57,
    62, 69, 61};
// [0]: SIGN -1, [1]: SIGN +1; entry L_out(k) = k mod 8 + 8 (k mod 11) holds
// (1/88) sum_j w_j exp(-2 pi i j k / 88)
__device__ double2 g_rader_w[2][88];

__global__ void rader_init_kernel()
{
    const int sgn = blockIdx.x ? 1 : -1, k = threadIdx.x;
    if (k >= 88) return;
    double re = 0.0, im = 0.0;
    int gj = 1;  // 3^j mod 89
    for (int j = 0; j < 88; j++) {
        double s1, c1, s2, c2;
        sincospi(2.0 * sgn * gj / 89.0, &s1, &c1);
        sincospi(-2.0 * ((j * k) % 88) / 88.0, &s2, &c2);
        re += c1 * c2 - s1 * s2;
        im += c1 * s2 + s1 * c2;
        gj = (gj * 3) % 89;
    }
    g_rader_w[blockIdx.x][k % 8 + 8 * (k % 11)] = make_double2(re / 88.0, im / 88.0);
}

template <int MODE, int NT>
__global__ void __launch_bounds__(NT, (NT == 128 ? 3 : 2)) pfa2047_alpha_kernel(CztArgs a)
{
    static_assert(MODE == CZT_ANA_ALPHA || MODE == CZT_SYN_ALPHA, "alpha stages only");
    constexpr int SIGN = MODE == CZT_ANA_ALPHA ? +1 : -1;
    extern __shared__ double2 smem[];
    // the row in layout d1 + 25 d2 (pitch 25: conflict-free shared-memory
    // access for the length-23 DFTs, two-way for the output gather); the 23
    // Rader convolutions in layout i + 9 j (pitch 103 per column: with the
    // work items (c1, j) taken c1-fastest, the gathers from the row, the
    // column stores and their reads back are conflict-free but for the
    // items where j changes)
    double2 *X = smem;
    double2 *Sc = smem + PFB_XS;
    double2 *X0 = Sc + 23 * PFB_SP;
    const int t = threadIdx.x;
    const int bl = a.bl, n = PFB_N;  // n = 2 bl - 1
    const int g = blockIdx.y, rr = blockIdx.x;
    pfa_load<MODE, NT, PFB_N>(a, X, [](int m) { return (m * 15) % 23 + PFB_P * ((m * 31) % 89); });
    __syncthreads();
    // length-23 DFTs along d1
    for (int d2 = t; d2 < 89; d2 += NT) {
        double2 x[23];
#pragma unroll
        for (int r = 0; r < 23; r++) x[r] = X[PFB_P * d2 + r];
        pfa_dft_out<23, SIGN>(x, X, PFB_P * d2, 1);
    }
    __syncthreads();
    // length-89 DFTs along d2 (column c1) by Rader: forward length-8 DFTs of
    // the permuted inputs
    for (int u = t; u < 23 * 11; u += NT) {
        const int c1 = u % 23, j = u / 23;
        double2 v[8];
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = X[c1 + PFB_P * c_rader_src[i + 8 * j]];
        Dft<8, -1>::run(v);
#pragma unroll
        for (int i = 0; i < 8; i++) Sc[c1 * PFB_SP + i + 9 * j] = v[i];
        if (j == 0) X0[c1] = X[c1];
    }
    __syncthreads();
    // forward length-11 DFTs, product with the DFT of w, inverse length-11
    for (int u = t; u < 23 * 8; u += NT) {
        const int c1 = u / 8, i = u % 8;
        double2 v[11];
#pragma unroll
        for (int jj = 0; jj < 11; jj++) v[jj] = Sc[c1 * PFB_SP + i + 9 * jj];
        pfa_dft<11, -1>(v);
        if (i == 0) X[c1] = cadd(X0[c1], v[0]);  // y_0 = x_0 + sum of the other inputs
#pragma unroll
        for (int kk = 0; kk < 11; kk++) v[kk] = cmul(v[kk], g_rader_w[SIGN > 0 ? 1 : 0][i + 8 * kk]);
        pfa_dft<11, +1>(v);
#pragma unroll
        for (int jj = 0; jj < 11; jj++) Sc[c1 * PFB_SP + i + 9 * jj] = v[jj];
    }
    __syncthreads();
    // inverse length-8 DFTs; y_{g^q} = x_0 + convolution
    for (int u = t; u < 23 * 11; u += NT) {
        const int c1 = u % 23, j = u / 23;
        double2 v[8];
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = Sc[c1 * PFB_SP + i + 9 * j];
        Dft<8, +1>::run(v);
        const double2 x0 = X0[c1];
#pragma unroll
        for (int i = 0; i < 8; i++) X[c1 + PFB_P * c_rader_dst[i + 8 * j]] = cadd(x0, v[i]);
    }
    __syncthreads();
    if (MODE == CZT_ANA_ALPHA) {
        for (int k = t; k < n; k += NT) {
            const double2 y = X[k % 23 + PFB_P * (k % 89)];
            double *p = a.out_r + (size_t)k + (size_t)n * (2 * rr + (size_t)2 * bl * g);
            p[0] = y.x;
            p[n] = y.y;
        }
    } else {
        const double hh = 0.5 * a.scale;
        for (int m = t; m < bl; m += NT) {
            const int mc = m == 0 ? 0 : n - m;
            const double2 Z = X[m % 23 + PFB_P * (m % 89)];
            const double2 Zc = cconj(X[mc % 23 + PFB_P * (mc % 89)]);
            const double2 sm = cadd(Z, Zc), d = csub(Z, Zc);
            st_pair(a.out_c + ((size_t)g * bl + m) * (2 * bl) + 2 * rr, make_double2(sm.x * hh, sm.y * hh),
                    make_double2(d.y * hh, -d.x * hh));
        }
    }
}

template <>
__device__ __forceinline__ void pfa_cs<3>(int j, double &c, double &s)
{
    constexpr double C[3] = {
        1.00000000000000000000, -0.500000000000000000000, -0.500000000000000000000};
    constexpr double S[3] = {
        0.0, 0.866025403784438646764, -0.866025403784438646764};
    c = C[j];
    s = S[j];
}
template <>
__device__ __forceinline__ void pfa_cs<31>(int j, double &c, double &s)
{
    constexpr double C[31] = {
        1.00000000000000000000, 0.979529941252494493938, 0.918957811620230629127, 0.820763441207276326364,
        0.688966919075686567801, 0.528964010326962457365, 0.347305252844820285542, 0.151427777504576663657,
        -0.050649168838712712279, -0.250652532258720539315, -0.440394151557634309516,
        -0.612105982547662844147, -0.758758122692790901913, -0.874346616144582118827,
        -0.954139256400048851476, -0.994869323391895146321, -0.994869323391895146321,
        -0.954139256400048851476, -0.874346616144582118827, -0.758758122692790901913,
        -0.612105982547662844147, -0.440394151557634309516, -0.250652532258720539315,
        -0.050649168838712712279, 0.151427777504576663657, 0.347305252844820285542, 0.528964010326962457365,
        0.688966919075686567801, 0.820763441207276326364, 0.918957811620230629127, 0.979529941252494493938};
    constexpr double S[31] = {
        0.0, 0.201298520088660079142, 0.394355855113318580102, 0.571268215094792279157,
        0.724792787229119958865, 0.848644257494750950464, 0.937752132147080458429, 0.988468324328111399162,
        0.998716507171052807146, 0.968077118866204305153, 0.897804539570741657137, 0.790775736937698582078,
        0.651372482722222207454, 0.485301962531081025215, 0.299363122973357954008, 0.101168321987432177786,
        -0.101168321987432177786, -0.299363122973357954008, -0.485301962531081025215,
        -0.651372482722222207454, -0.790775736937698582078, -0.897804539570741657137,
        -0.968077118866204305153, -0.998716507171052807146, -0.988468324328111399162,
        -0.937752132147080458429, -0.848644257494750950464, -0.724792787229119958865,
        -0.571268215094792279157, -0.394355855113318580102, -0.201298520088660079142};
    c = C[j];
    s = S[j];
}

// ---------------------------------------------------------------------------
// Prime-factor alpha stages at bl = 256: n = 511 = 7 * 73
//
// As at bl = 1024 with 23 x 89 replaced by 7 x 73: row layout d1 + 9 d2 (input
// digits (5n) mod 7, (21n) mod 73), length-7 DFTs along d1, and the length-73
// DFTs by Rader's algorithm with the primitive root 5: a cyclic convolution of
// length 72 = 8 x 9 (radix 8 in registers, then length 9; layout L = i + 8 j
// with input digits q mod 8, (8q) mod 9), the product with the DFT of
// w_j = exp(SIGN 2 pi i 5^j / 73) (g_rader73_w, built with the length-89 table
// by pfa_prepare), and the inverse.
// ---------------------------------------------------------------------------
constexpr int PFD_N = 511;
constexpr int PFD_P = 9;               // pitch of d2 in the shared row
constexpr int PFD_XS = PFD_P * 73;
constexpr int PFD_SP = 83;             // pitch of a Rader column (positions i + 9 j, i < 8, j < 9)
constexpr int PFD_THREADS = 128;

__constant__ int c_rader73_src[72] = {
    1, 22, 46, 63, 72, 51, 27, 10, 37, 11, 23, 68, 36, 62, 50, 5, 55, 42, 48, 34, 18, 31, 25, 39, 64, 21, 24, 17,
    9, 52, 49, 56, 32, 47, 12, 45, 41, 26, 61, 28, 16, 60, 6, 59, 57, 13, 67, 14, 8, 30, 3, 66, 65, 43, 70, 7, 4,
    15, 38, 33, 69, 58, 35, 40, 2, 44, 19, 53, 71, 29, 54, 20};
__constant__ int c_rader73_dst[72] = {
    1, 10, 27, 51, 72, 63, 46, 22, 2, 20, 54, 29, 71, 53, 19, 44, 4, 40, 35, 58, 69, 33, 38, 15, 8, 7, 70, 43, 65,
    66, 3, 30, 16, 14, 67, 13, 57, 59, 6, 60, 32, 28, 61, 26, 41, 45, 12, 47, 64, 56, 49, 52, 9, 17, 24, 21, 55,
    39, 25, 31, 18, 34, 48, 42, 37, 5, 50, 62, 36, 68, 23, 11};
// [0]: SIGN -1, [1]: SIGN +1; entry k mod 8 + 8 (k mod 9) holds
// (1/72) sum_j w_j exp(-2 pi i j k / 72)
__device__ double2 g_rader73_w[2][72];

__global__ void rader73_init_kernel()
{
    const int sgn = blockIdx.x ? 1 : -1, k = threadIdx.x;
    if (k >= 72) return;
    double re = 0.0, im = 0.0;
    int gj = 1;  // 5^j mod 73
    for (int j = 0; j < 72; j++) {
        double s1, c1, s2, c2;
        sincospi(2.0 * sgn * gj / 73.0, &s1, &c1);
        sincospi(-2.0 * ((j * k) % 72) / 72.0, &s2, &c2);
        re += c1 * c2 - s1 * s2;
        im += c1 * s2 + s1 * c2;
        gj = (gj * 5) % 73;
    }
    g_rader73_w[blockIdx.x][k % 8 + 8 * (k % 9)] = make_double2(re / 72.0, im / 72.0);
}

template <int MODE>
__global__ void __launch_bounds__(PFD_THREADS) pfa511_alpha_kernel(CztArgs a)
{
    static_assert(MODE == CZT_ANA_ALPHA || MODE == CZT_SYN_ALPHA, "alpha stages only");
    constexpr int SIGN = MODE == CZT_ANA_ALPHA ? +1 : -1;
    constexpr int NT = PFD_THREADS;
    extern __shared__ double2 smem[];
    double2 *X = smem;
    double2 *Sc = smem + PFD_XS;
    double2 *X0 = Sc + 7 * PFD_SP;
    const int t = threadIdx.x;
    const int bl = a.bl, n = PFD_N;  // n = 2 bl - 1
    const int g = blockIdx.y, rr = blockIdx.x;
    pfa_load<MODE, NT, PFD_N>(a, X, [](int m) { return (m * 5) % 7 + PFD_P * ((m * 21) % 73); });
    __syncthreads();
    // length-7 DFTs along d1
    for (int d2 = t; d2 < 73; d2 += NT) {
        double2 x[7];
#pragma unroll
        for (int r = 0; r < 7; r++) x[r] = X[PFD_P * d2 + r];
        pfa_dft_out<7, SIGN>(x, X, PFD_P * d2, 1);
    }
    __syncthreads();
    // length-73 DFTs along d2 (column c1) by Rader: forward length-8 DFTs
    for (int u = t; u < 7 * 9; u += NT) {
        const int c1 = u % 7, j = u / 7;
        double2 v[8];
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = X[c1 + PFD_P * c_rader73_src[i + 8 * j]];
        Dft<8, -1>::run(v);
#pragma unroll
        for (int i = 0; i < 8; i++) Sc[c1 * PFD_SP + i + 9 * j] = v[i];
        if (j == 0) X0[c1] = X[c1];
    }
    __syncthreads();
    // forward length-9 DFTs, product with the DFT of w, inverse length-9
    for (int u = t; u < 7 * 8; u += NT) {
        const int c1 = u / 8, i = u % 8;
        double2 v[9];
#pragma unroll
        for (int jj = 0; jj < 9; jj++) v[jj] = Sc[c1 * PFD_SP + i + 9 * jj];
        pfa_dft<9, -1>(v);
        if (i == 0) X[c1] = cadd(X0[c1], v[0]);  // y_0 = x_0 + sum of the other inputs
#pragma unroll
        for (int kk = 0; kk < 9; kk++) v[kk] = cmul(v[kk], g_rader73_w[SIGN > 0 ? 1 : 0][i + 8 * kk]);
        pfa_dft<9, +1>(v);
#pragma unroll
        for (int jj = 0; jj < 9; jj++) Sc[c1 * PFD_SP + i + 9 * jj] = v[jj];
    }
    __syncthreads();
    // inverse length-8 DFTs; y_{g^q} = x_0 + convolution
    for (int u = t; u < 7 * 9; u += NT) {
        const int c1 = u % 7, j = u / 7;
        double2 v[8];
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = Sc[c1 * PFD_SP + i + 9 * j];
        Dft<8, +1>::run(v);
        const double2 x0 = X0[c1];
#pragma unroll
        for (int i = 0; i < 8; i++) X[c1 + PFD_P * c_rader73_dst[i + 8 * j]] = cadd(x0, v[i]);
    }
    __syncthreads();
    if (MODE == CZT_ANA_ALPHA) {
        for (int k = t; k < n; k += NT) {
            const double2 y = X[k % 7 + PFD_P * (k % 73)];
            double *p = a.out_r + (size_t)k + (size_t)n * (2 * rr + (size_t)2 * bl * g);
            p[0] = y.x;
            p[n] = y.y;
        }
    } else {
        const double hh = 0.5 * a.scale;
        for (int m = t; m < bl; m += NT) {
            const int mc = m == 0 ? 0 : n - m;
            const double2 Z = X[m % 7 + PFD_P * (m % 73)];
            const double2 Zc = cconj(X[mc % 7 + PFD_P * (mc % 73)]);
            const double2 sm = cadd(Z, Zc), d = csub(Z, Zc);
            st_pair(a.out_c + ((size_t)g * bl + m) * (2 * bl) + 2 * rr, make_double2(sm.x * hh, sm.y * hh),
                    make_double2(d.y * hh, -d.x * hh));
        }
    }
}

// ---------------------------------------------------------------------------
// Prime-factor alpha stages at bl = 512: n = 1023 = 3 * 11 * 31
//
// Good-Thomas as at bl = 2048 (layout L = d1 + 3 d2 + 33 d3, input digits
// (n u_i) mod R_i with u_i = (1023/R_i)^-1 mod R_i = 2, 9, 16, output k at
// digits k mod R_i), DFTs of length 3 and 11 in place, then the length-31 DFTs
// written straight to their output positions (pfa_dft_out keeps their
// registers to about 31 complex values).  About 45 FP64 operations per point
// against ~220 for the 2048-point Bluestein convolution.
// ---------------------------------------------------------------------------
constexpr int PFC_N = 1023, PFC_THREADS = 128;

__device__ __forceinline__ int pfc_in_pos(int n) { return (n * 2) % 3 + 3 * ((n * 9) % 11) + 33 * ((n * 16) % 31); }
__device__ __forceinline__ int pfc_out_pos(int k) { return k % 3 + 3 * (k % 11) + 33 * (k % 31); }

// in-place DFTs of length R along stride S of the 1023-point layout
template <int R, int S, int SIGN>
__device__ __forceinline__ void pfc_stage(double2 *sm, int t)
{
    for (int d = t; d < PFC_N / R; d += PFC_THREADS) {
        const int base = (d % S) + (d / S) * (S * R);
        double2 x[R];
#pragma unroll
        for (int r = 0; r < R; r++) x[r] = sm[base + r * S];
        pfa_dft<R, SIGN>(x);
#pragma unroll
        for (int r = 0; r < R; r++) sm[base + r * S] = x[r];
    }
}

template <int MODE>
__global__ void __launch_bounds__(PFC_THREADS, 3) pfa1023_alpha_kernel(CztArgs a)
{
    static_assert(MODE == CZT_ANA_ALPHA || MODE == CZT_SYN_ALPHA, "alpha stages only");
    constexpr int SIGN = MODE == CZT_ANA_ALPHA ? +1 : -1;
    extern __shared__ double2 smem[];
    const int t = threadIdx.x;
    const int bl = a.bl, n = PFC_N;  // n = 2 bl - 1
    const int g = blockIdx.y, rr = blockIdx.x;
    pfa_load<MODE, PFC_THREADS, PFC_N>(a, smem, [](int m) { return pfc_in_pos(m); });
    __syncthreads();
    pfc_stage<3, 1, SIGN>(smem, t);
    __syncthreads();
    pfc_stage<11, 3, SIGN>(smem, t);
    __syncthreads();
    // length-31 DFTs along d3 (stride 33), in registers, back to the same positions
    for (int d = t; d < 33; d += PFC_THREADS) {
        double2 x[31];
#pragma unroll
        for (int r = 0; r < 31; r++) x[r] = smem[d + 33 * r];
        pfa_dft_out<31, SIGN>(x, smem, d, 33);
    }
    __syncthreads();
    if (MODE == CZT_ANA_ALPHA) {
        for (int k = t; k < n; k += PFC_THREADS) {
            const double2 y = smem[pfc_out_pos(k)];
            double *p = a.out_r + (size_t)k + (size_t)n * (2 * rr + (size_t)2 * bl * g);
            p[0] = y.x;
            p[n] = y.y;
        }
    } else {
        const double hh = 0.5 * a.scale;
        for (int m = t; m < bl; m += PFC_THREADS) {
            const double2 Z = smem[pfc_out_pos(m)];
            const double2 Zc = cconj(smem[pfc_out_pos(m == 0 ? 0 : n - m)]);
            const double2 sm = cadd(Z, Zc), d = csub(Z, Zc);
            st_pair(a.out_c + ((size_t)g * bl + m) * (2 * bl) + 2 * rr, make_double2(sm.x * hh, sm.y * hh),
                    make_double2(d.y * hh, -d.x * hh));
        }
    }
}

template <>
__device__ __forceinline__ void pfa_cs<17>(int j, double &c, double &s)
{
    constexpr double C[17] = {
        1.00000000000000000000, 0.932472229404355804573, 0.739008917220659115925, 0.445738355776538267396,
        0.092268359463301995240, -0.273662990072082863539, -0.602634636379256389179, -0.850217135729614152134,
        -0.982973099683901778282, -0.982973099683901778282, -0.850217135729614152134, -0.602634636379256389179,
        -0.273662990072082863539, 0.092268359463301995240, 0.445738355776538267396, 0.739008917220659115925,
        0.932472229404355804573};
    constexpr double S[17] = {
        0.0, 0.361241666187152948745, 0.673695643646557211713, 0.895163291355062322067, 0.995734176295034521871,
        0.961825643172819070409, 0.798017227280239503333, 0.526432162877355800245, 0.183749517816570331574,
        -0.183749517816570331574, -0.526432162877355800245, -0.798017227280239503333, -0.961825643172819070409,
        -0.995734176295034521871, -0.895163291355062322067, -0.673695643646557211713, -0.361241666187152948745};
    c = C[j];
    s = S[j];
}

// ---------------------------------------------------------------------------
// Prime-factor alpha stages of the small scales: n = 2bl - 1 = R1 R2 R3 with
// small pairwise coprime factors (bl = 2: 3; 4: 7; 8: 3 * 5; 16: 31; 32: 7 * 9;
// 128: 3 * 5 * 17), Good-Thomas with direct symmetric-pair DFTs (factors of 1
// are skipped), one CTA per row pair as the kernels above.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int pfs_inv(int a, int r)
{
    int x = 1;
    while (r > 1 && (a * x) % r != 1) x++;
    return x;
}

template <int N, int R, int S>
__device__ __forceinline__ void pfs_stage(double2 *sm, int t, int nt, int sign)
{
    for (int d = t; d < N / R; d += nt) {
        const int base = (d % S) + (d / S) * (S * R);
        double2 x[R];
#pragma unroll
        for (int r = 0; r < R; r++) x[r] = sm[base + r * S];
        if (sign > 0) pfa_dft<R, +1>(x);
        else pfa_dft<R, -1>(x);
#pragma unroll
        for (int r = 0; r < R; r++) sm[base + r * S] = x[r];
    }
}

constexpr int PFS_THREADS = 64;

template <int R1, int R2, int R3, int MODE>
__global__ void __launch_bounds__(PFS_THREADS) pfs_alpha_kernel(CztArgs a)
{
    static_assert(MODE == CZT_ANA_ALPHA || MODE == CZT_SYN_ALPHA, "alpha stages only");
    constexpr int SIGN = MODE == CZT_ANA_ALPHA ? +1 : -1;
    constexpr int N = R1 * R2 * R3, NT = PFS_THREADS;
    constexpr int U1 = pfs_inv((N / R1) % R1, R1), U2 = pfs_inv((N / R2) % R2, R2), U3 = pfs_inv((N / R3) % R3, R3);
    extern __shared__ double2 smem[];
    const int t = threadIdx.x;
    const int bl = a.bl, n = N;  // n = 2 bl - 1
    const int g = blockIdx.y, rr = blockIdx.x;
    pfa_load<MODE, NT, N>(a, smem, [](int m) {
        return (m * U1) % R1 + R1 * ((m * U2) % R2) + R1 * R2 * ((m * U3) % R3);
    });
    __syncthreads();
    if constexpr (R1 > 1) pfs_stage<N, R1, 1>(smem, t, NT, SIGN);
    __syncthreads();
    if constexpr (R2 > 1) {
        pfs_stage<N, R2, R1>(smem, t, NT, SIGN);
        __syncthreads();
    }
    if constexpr (R3 > 1) {
        pfs_stage<N, R3, R1 * R2>(smem, t, NT, SIGN);
        __syncthreads();
    }
    auto opos = [](int k) { return k % R1 + R1 * (k % R2) + R1 * R2 * (k % R3); };
    if (MODE == CZT_ANA_ALPHA) {
        for (int k = t; k < n; k += NT) {
            const double2 y = smem[opos(k)];
            double *p = a.out_r + (size_t)k + (size_t)n * (2 * rr + (size_t)2 * bl * g);
            p[0] = y.x;
            p[n] = y.y;
        }
    } else {
        const double hh = 0.5 * a.scale;
        for (int m = t; m < bl; m += NT) {
            const double2 Z = smem[opos(m)];
            const double2 Zc = cconj(smem[opos(m == 0 ? 0 : n - m)]);
            const double2 sm = cadd(Z, Zc), d = csub(Z, Zc);
            st_pair(a.out_c + ((size_t)g * bl + m) * (2 * bl) + 2 * rr, make_double2(sm.x * hh, sm.y * hh),
                    make_double2(d.y * hh, -d.x * hh));
        }
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

__global__ void combine_kernel(CombineArgs a)
{
    const int B = a.B;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)B * B;
         i += (long long)gridDim.x * blockDim.x) {
        const int l = (int)(i % B), m = (int)(i / B);
        double2 f = make_double2(0.0, 0.0);
        if (m <= l) {
            for (int j = 0; j <= a.J; j++)
                if (l > a.blo[j] && l < a.bl[j]) f = cadd(f, a.parts[a.off[j] + (size_t)(l - a.blo[j] - 1) * a.bl[j] + m]);
        }
        if (l < a.bs && m < a.bs) f = cadd(f, cscale(a.scoeff[l + (size_t)a.bs * m], a.Phi2[l]));
        a.flm[i] = f;
    }
}

// ===========================================================================
// Launchers
// ===========================================================================
template <int NP, int S, int MINB>
static int launch_lwalk_np(const LwalkArgs &a, cudaStream_t s)
{
    using L = LwalkSmem<NP, S>;
    static bool attr[64] = {false};
    int dev = 0;
    S2DW_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 64 && !attr[dev]) {
        if (MINB > 0)
            S2DW_CUDA_TRY(cudaFuncSetAttribute(lwalk_kernel_minb<NP, S, (MINB > 0 ? MINB : 1)>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::BYTES));
        else
            S2DW_CUDA_TRY(cudaFuncSetAttribute(lwalk_kernel<NP, S, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)L::BYTES));
        attr[dev] = true;
    }
    if (a.ntiles <= 0) return S2DWC_OK;
    if (MINB > 0)
        lwalk_kernel_minb<NP, S, (MINB > 0 ? MINB : 1)><<<a.ntiles, LW_W * 32, L::BYTES, s>>>(a);
    else
        lwalk_kernel<NP, S, 0><<<a.ntiles, LW_W * 32, L::BYTES, s>>>(a);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

static int g_lwalk_variant = 0, g_mwalk_variant = 0;

int lwalk_tile_m(int NP) { return LW_W * (NP > 4 ? 2 : 4); }  // pairs per thread: 4, or 2 for N > 8
// the two-l-per-thread synthesis kernel (the default, variant 4), for N <= 8
// (NP <= 4; 4 m per thread for NP <= 2, 2 for NP = 3, 4); measured on B200 at
// B=1024, N=4: 343 -> 322 us per full-band launch, FP64 pipe 49 -> 61 %,
// shared-memory wavefronts 61 -> 43 % of peak
static bool mwalk2_used(int NP) { return g_mwalk_variant == 4 && NP <= 4; }
static int mwalk2_qm(int NP) { return NP <= 2 ? 4 : 2; }
int mwalk_tile_m(int NP)
{
    if (mwalk2_used(NP)) return MW_W * mwalk2_qm(NP);
    return MW_W * (g_mwalk_variant == 1 && NP <= 4 ? 8 : 4);
}
int mwalk_tile_l(int NP) { return mwalk2_used(NP) ? M2_TL : 32; }

void build_lwalk_tiles(int bl, int blo, int ws, std::vector<int2> &t)
{
    // work of tile (pt, mt): walk from max(p0, m0) to bl-1
    t.clear();
    const int tp = (bl + 31) / 32, tm = (bl + ws - 1) / ws;
    for (int pt = 0; pt < tp; pt++)
        for (int mt = 0; mt < tm; mt++) t.push_back(make_int2(pt, mt));
    std::stable_sort(t.begin(), t.end(), [ws](int2 a, int2 b) {
        return std::max(a.x * 32, a.y * ws) < std::max(b.x * 32, b.y * ws);
    });
    (void)blo;
}

void build_mwalk_tiles(int bl, int blo, int wq, int th, std::vector<int2> &t)
{
    // tile (lt, mt) covers l in [blo+1+th lt, +th), m in [wq mt, +wq); its
    // walk length is ~ the largest l; tiles entirely above m <= l are dropped
    t.clear();
    const int nl = bl - blo - 1;
    if (nl <= 0) return;
    const int tl = (nl + th - 1) / th, tm = (bl + wq - 1) / wq;
    for (int lt = tl - 1; lt >= 0; lt--) {
        const int lmax = std::min(blo + 1 + lt * th + th - 1, bl - 1);
        for (int mt = 0; mt < tm; mt++)
            if (mt * wq <= lmax) t.push_back(make_int2(lt, mt));
    }
}
void set_walk_variants(int lw, int mw)
{
    g_lwalk_variant = lw;
    g_mwalk_variant = mw;
}

template <int S, int MINB>
static int launch_lwalk_s(const LwalkArgs &a, cudaStream_t s)
{
    switch (a.NP) {
    case 1: return launch_lwalk_np<1, S, MINB>(a, s);
    case 2: return launch_lwalk_np<2, S, MINB>(a, s);
    case 3: return launch_lwalk_np<3, S, MINB>(a, s);
    case 4: return launch_lwalk_np<4, S, MINB>(a, s);
    // N > 8: two pairs per thread keep the accumulators in registers
    case 5: return launch_lwalk_np<5, 2, 0>(a, s);
    case 6: return launch_lwalk_np<6, 2, 0>(a, s);
    case 7: return launch_lwalk_np<7, 2, 0>(a, s);
    case 8: return launch_lwalk_np<8, 2, 0>(a, s);
    }
    return set_error(S2DWC_ERROR_SIZE_INVALID, "lwalk: unsupported N=%d (N<=%d)", a.N, S2DW_NMAX);
}

int launch_lwalk(const LwalkArgs &a, cudaStream_t s)
{
    switch (g_lwalk_variant) {
    case 1: return launch_lwalk_s<4, 4>(a, s);
    case 2: return launch_lwalk_s<4, 3>(a, s);
    default:
        // more resident CTAs where the register cap costs no spills and the
        // grid is many waves deep (bl >= 1024: 2048+ tiles); measured on
        // B200: NP = 2, bl = 1024: 3 CTAs/SM 10 % faster than 2; NP = 1:
        // 4 CTAs/SM 4 % faster.  Smaller grids lose more to the tail wave,
        // and NP >= 3 spills under the caps.
        if (a.bl >= 1024 && a.NP == 2) return launch_lwalk_np<2, 4, 3>(a, s);
        if (a.bl >= 1024 && a.NP == 1) return launch_lwalk_np<1, 4, 4>(a, s);
        return launch_lwalk_s<4, 0>(a, s);
    }
}

template <int NP, int Q, int MINB>
static int launch_mwalk_np(const MwalkArgs &a, cudaStream_t s)
{
    using L = MwalkSmem<NP, Q>;
    const int nl = a.bl - a.blo - 1;
    if (nl <= 0) return S2DWC_OK;
    static bool attr[64] = {false};
    int dev = 0;
    S2DW_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 64 && !attr[dev]) {
        if (MINB > 0)
            S2DW_CUDA_TRY(cudaFuncSetAttribute(mwalk_kernel_minb<NP, Q, (MINB > 0 ? MINB : 1)>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::BYTES));
        else
            S2DW_CUDA_TRY(cudaFuncSetAttribute(mwalk_kernel<NP, Q, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)L::BYTES));
        attr[dev] = true;
    }
    if (a.ntiles <= 0) return S2DWC_OK;
    if (MINB > 0)
        mwalk_kernel_minb<NP, Q, (MINB > 0 ? MINB : 1)><<<a.ntiles, MW_W * 32, L::BYTES, s>>>(a);
    else
        mwalk_kernel<NP, Q, 0><<<a.ntiles, MW_W * 32, L::BYTES, s>>>(a);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

template <int NP, int QM>
static int launch_mwalk2(const MwalkArgs &a, cudaStream_t s)
{
    using L = Mwalk2Smem<NP, QM>;
    if (a.bl - a.blo - 1 <= 0 || a.ntiles <= 0) return S2DWC_OK;
    if (!a.GT) return set_error(S2DWC_ERROR_ARG_INVALID, "mwalk2: transposed tables missing");
    static bool attr[64] = {false};
    int dev = 0;
    S2DW_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 64 && !attr[dev]) {
        S2DW_CUDA_TRY(cudaFuncSetAttribute(mwalk2_kernel<NP, QM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)L::BYTES));
        attr[dev] = true;
    }
    mwalk2_kernel<NP, QM><<<a.ntiles, MW_W * 32, L::BYTES, s>>>(a);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

int launch_gsyn_t(const GsTArgs &a, cudaStream_t s)
{
    const long long total = (long long)a.rows * (a.NP + 1) * a.Ts;
    if (total <= 0) return S2DWC_OK;
    long long blocks = (total + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    gsyn_t_kernel<<<(int)blocks, 256, 0, s>>>(a);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

template <int Q, int MINB>
static int launch_mwalk_q(const MwalkArgs &a, cudaStream_t s)
{
    switch (a.NP) {
    case 1: return launch_mwalk_np<1, Q, MINB>(a, s);
    case 2: return launch_mwalk_np<2, Q, MINB>(a, s);
    case 3: return launch_mwalk_np<3, Q, MINB>(a, s);
    case 4: return launch_mwalk_np<4, Q, MINB>(a, s);
    // N > 8: no register cap (the G rows of 5-8 n values stay in registers)
    case 5: return launch_mwalk_np<5, 4, 0>(a, s);
    case 6: return launch_mwalk_np<6, 4, 0>(a, s);
    case 7: return launch_mwalk_np<7, 4, 0>(a, s);
    case 8: return launch_mwalk_np<8, 4, 0>(a, s);
    }
    return set_error(S2DWC_ERROR_SIZE_INVALID, "mwalk: unsupported N=%d (N<=%d)", a.N, S2DW_NMAX);
}

int launch_mwalk(const MwalkArgs &a, cudaStream_t s)
{
    // the kernel follows the plan's tile shape
    if (a.tile_l == M2_TL) {
        if (a.NP > 4 || a.tile_m != MW_W * mwalk2_qm(a.NP))
            return set_error(S2DWC_ERROR_ARG_INVALID, "mwalk: tile shape %dx%d for NP=%d", a.tile_l, a.tile_m, a.NP);
        switch (a.NP) {
        case 1: return launch_mwalk2<1, 4>(a, s);
        case 2: return launch_mwalk2<2, 4>(a, s);
        case 3: return launch_mwalk2<3, 2>(a, s);
        default: return launch_mwalk2<4, 2>(a, s);
        }
    }
    if (a.tile_l != 32) return set_error(S2DWC_ERROR_ARG_INVALID, "mwalk: tile height %d", a.tile_l);
    if (a.tile_m == MW_W * 8) return launch_mwalk_q<8, 0>(a, s);
    switch (g_mwalk_variant) {
    case 2: return launch_mwalk_q<4, 5>(a, s);
    case 3: return launch_mwalk_q<4, 4>(a, s);
    // 3 CTAs/SM (<= 168 registers, no spills): 3-10 % faster than 4 CTAs/SM
    // with 128 registers and small spills, at N = 1, 3, 4, 6, 8 (B200)
    default: return launch_mwalk_q<4, 3>(a, s);
    }
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

template <int V, int THREADS, int MODE>
static int launch_fft_t(const CztArgs &a, cudaStream_t s)
{
    constexpr int E = V * THREADS;
    const int M = a.czt.M, R = E / M;
    const int nhi = (M + 63) / 64;
    const size_t smem = sizeof(double2) * ((size_t)padix(E) + 1 + nhi + 64 + S2DW_NPMAX * S2DW_NMAX);  // + ph[q][g]
    static bool attr[64] = {false};
    int dev = 0;
    S2DW_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 64 && !attr[dev]) {
        S2DW_CUDA_TRY(cudaFuncSetAttribute(fft_kernel<V, THREADS, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)(sizeof(double2) * ((size_t)padix(E) + 1 + 128 + 64 + S2DW_NPMAX * S2DW_NMAX))));
        attr[dev] = true;
    }
    const int grid = (a.rows + R - 1) / R;
    if (grid == 0) return S2DWC_OK;
    fft_kernel<V, THREADS, MODE><<<grid, THREADS, smem, s>>>(a);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

template <int V, int THREADS>
static int launch_fft_mode(const CztArgs &a, cudaStream_t s)
{
    switch (a.mode) {
    case CZT_ANA_BETA: return launch_fft_t<V, THREADS, CZT_ANA_BETA>(a, s);
    case CZT_ANA_ALPHA: return launch_fft_t<V, THREADS, CZT_ANA_ALPHA>(a, s);
    case CZT_SYN_ALPHA: return launch_fft_t<V, THREADS, CZT_SYN_ALPHA>(a, s);
    case CZT_SYN_BETA: return launch_fft_t<V, THREADS, CZT_SYN_BETA>(a, s);
    case FFT_ANA_BETA: return launch_fft_t<V, THREADS, FFT_ANA_BETA>(a, s);
    case FFT_SYN_BETA: return launch_fft_t<V, THREADS, FFT_SYN_BETA>(a, s);
    }
    return set_error(S2DWC_ERROR_ARG_INVALID, "unknown transform mode %d", a.mode);
}

template <int MODE, int LGM>
static int launch_large_t(const CztArgs &a, cudaStream_t s)
{
    constexpr int M = 1 << LGM;
    const size_t smem = sizeof(double2) * ((size_t)padix(M) + 1 + M / 64 + 64 + S2DW_NMAX);  // + phases ph[g], g < N
    static bool attr[64] = {false};
    int dev = 0;
    S2DW_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 64 && !attr[dev]) {
        S2DW_CUDA_TRY(cudaFuncSetAttribute(fft_large_kernel<MODE, LGM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
        attr[dev] = true;
    }
    // rows are (g or q) x (m or b pair); every mode has bl rows per g
    const int ng = a.rows / a.bl;
    constexpr bool synb = (MODE == CZT_SYN_BETA || MODE == FFT_SYN_BETA);
    const dim3 grid = synb ? dim3(ng, a.bl) : dim3(a.bl, ng);
    fft_large_kernel<MODE, LGM><<<grid, M / 16, smem, s>>>(a);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

template <int LGM>
static int launch_large(const CztArgs &a, cudaStream_t s)
{
    switch (a.mode) {
    case CZT_ANA_BETA: return launch_large_t<CZT_ANA_BETA, LGM>(a, s);
    case CZT_ANA_ALPHA: return launch_large_t<CZT_ANA_ALPHA, LGM>(a, s);
    case CZT_SYN_ALPHA: return launch_large_t<CZT_SYN_ALPHA, LGM>(a, s);
    case CZT_SYN_BETA: return launch_large_t<CZT_SYN_BETA, LGM>(a, s);
    case FFT_ANA_BETA: return launch_large_t<FFT_ANA_BETA, LGM>(a, s);
    case FFT_SYN_BETA: return launch_large_t<FFT_SYN_BETA, LGM>(a, s);
    }
    return set_error(S2DWC_ERROR_ARG_INVALID, "unknown transform mode %d", a.mode);
}

template <int R1, int R2, int R3, int MODE>
static int launch_pfs(const CztArgs &a, cudaStream_t s)
{
    const size_t smem = sizeof(double2) * (R1 * R2 * R3);
    const dim3 grid(a.bl, a.rows / a.bl);  // (b pair, g)
    pfs_alpha_kernel<R1, R2, R3, MODE><<<grid, PFS_THREADS, smem, s>>>(a);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}
template <int R1, int R2, int R3>
static int launch_pfs_m(const CztArgs &a, cudaStream_t s)
{
    return a.mode == CZT_ANA_ALPHA ? launch_pfs<R1, R2, R3, CZT_ANA_ALPHA>(a, s)
                                   : launch_pfs<R1, R2, R3, CZT_SYN_ALPHA>(a, s);
}

template <int MODE>
static int launch_pfa511(const CztArgs &a, cudaStream_t s)
{
    const size_t smem = sizeof(double2) * (PFD_XS + 7 * PFD_SP + 7);  // 20 KB: no opt-in needed
    const dim3 grid(a.bl, a.rows / a.bl);                              // (b pair, g)
    pfa511_alpha_kernel<MODE><<<grid, PFD_THREADS, smem, s>>>(a);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

template <int MODE>
static int launch_pfa1023(const CztArgs &a, cudaStream_t s)
{
    const size_t smem = sizeof(double2) * PFC_N;  // 16 KB: no opt-in needed
    const dim3 grid(a.bl, a.rows / a.bl);          // (b pair, g)
    pfa1023_alpha_kernel<MODE><<<grid, PFC_THREADS, smem, s>>>(a);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

template <int MODE>
static int launch_pfa(const CztArgs &a, cudaStream_t s)
{
    const size_t smem = sizeof(double2) * PFA_N;
    static bool attr[64] = {false};
    int dev = 0;
    S2DW_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 64 && !attr[dev]) {
        S2DW_CUDA_TRY(cudaFuncSetAttribute(pfa_alpha_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
        attr[dev] = true;
    }
    const dim3 grid(a.bl, a.rows / a.bl);  // (b pair, g)
    pfa_alpha_kernel<MODE><<<grid, PFA_THREADS, smem, s>>>(a);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

template <int MODE, int NT>
static int launch_pfa2047(const CztArgs &a, cudaStream_t s)
{
    const size_t smem = sizeof(double2) * (PFB_XS + 23 * PFB_SP + 23);
    static bool attr[64] = {false};
    int dev = 0;
    S2DW_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 64 && !attr[dev]) {
        S2DW_CUDA_TRY(cudaFuncSetAttribute(pfa2047_alpha_kernel<MODE, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
        attr[dev] = true;
    }
    const dim3 grid(a.bl, a.rows / a.bl);  // (b pair, g)
    pfa2047_alpha_kernel<MODE, NT><<<grid, NT, smem, s>>>(a);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

static bool g_rader_ready[64] = {false};

int pfa_prepare()
{
    int dev = 0;
    S2DW_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(S2DWC_ERROR_ARG_INVALID, "device index %d", dev);
    if (g_rader_ready[dev]) return S2DWC_OK;
    rader_init_kernel<<<2, 96>>>();
    S2DW_CUDA_TRY(cudaGetLastError());
    rader73_init_kernel<<<2, 96>>>();
    S2DW_CUDA_TRY(cudaGetLastError());
    S2DW_CUDA_TRY(cudaStreamSynchronize(0));
    g_rader_ready[dev] = true;
    return S2DWC_OK;
}

static bool g_pfa = true;  // prime-factor alpha stages at bl = 2048, 1024, 512 and 256
static bool g_pfa1023 = true;  // bl = 512 (measurement switch)
static bool g_pfa511 = true;   // bl = 256 (measurement switch)
static bool g_pfa_small = true;  // bl = 2 .. 128 except 64 (measurement switch)
void set_pfa_small(bool on) { g_pfa_small = on; }
void set_pfa1023(bool on) { g_pfa1023 = on; }
void set_pfa511(bool on) { g_pfa511 = on; }
static int g_pfa2047_threads = 128;
void set_pfa(bool on) { g_pfa = on; }
void set_pfa2047_threads(int n) { g_pfa2047_threads = n == 256 ? 256 : 128; }

static int g_fft_values = 8;  // values per thread of the general FFT engine (8 or 16)
static bool g_large_2048 = true;  // M = 2048 transforms on the one-row-per-CTA engines
static bool g_alpha_prefetch = true;  // contiguous-input stages: persistent kernel with prefetched input

// Persistent launch of the prefetching stages: as many CTAs as fit on the
// device at once, each looping over rows.
template <int MODE, int LGM>
static int launch_pf(const CztArgs &a, cudaStream_t s)
{
    constexpr int M = 1 << LGM, THREADS = M / 16;
    const int chunks = pf_chunks<MODE>(a.bl);
    if (chunks > M) return set_error(S2DWC_ERROR_SIZE_INVALID, "prefetch stage: bl=%d does not fit M=%d", a.bl, M);
    const size_t smem = sizeof(double2) * ((size_t)padix(M) + 1 + M / 64 + 64 + (size_t)chunks);
    static int resident[64] = {0};
    static size_t smem_set[64] = {0};
    int dev = 0;
    S2DW_CUDA_TRY(cudaGetDevice(&dev));
    if (dev >= 64) return set_error(S2DWC_ERROR_ARG_INVALID, "device index %d", dev);
    if (smem_set[dev] < smem) {
        S2DW_CUDA_TRY(cudaFuncSetAttribute(fft_pf_kernel<MODE, LGM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
        int per_sm = 0, sms = 0;
        S2DW_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fft_pf_kernel<MODE, LGM>, THREADS, smem));
        S2DW_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        resident[dev] = std::max(1, per_sm) * sms;
        smem_set[dev] = smem;
    }
    const int grid = std::min(a.rows, resident[dev]);
    if (grid <= 0) return S2DWC_OK;
    fft_pf_kernel<MODE, LGM><<<grid, THREADS, smem, s>>>(a);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

void set_alpha_prefetch(bool on) { g_alpha_prefetch = on; }

int launch_czt(const CztArgs &a, cudaStream_t s)
{
    if (g_pfa && g_pfa_small && (a.mode == CZT_ANA_ALPHA || a.mode == CZT_SYN_ALPHA) && a.rows % a.bl == 0) {
        switch (a.bl) {
        case 2: return launch_pfs_m<3, 1, 1>(a, s);
        case 4: return launch_pfs_m<7, 1, 1>(a, s);
        case 8: return launch_pfs_m<3, 5, 1>(a, s);
        case 16: return launch_pfs_m<31, 1, 1>(a, s);
        case 32: return launch_pfs_m<7, 9, 1>(a, s);
        case 128: return launch_pfs_m<3, 5, 17>(a, s);
        default: break;
        }
    }
    if (g_pfa && g_pfa511 && a.bl == 256 && 2 * a.bl - 1 == PFD_N && a.rows % a.bl == 0) {
        int dev = 0;
        S2DW_CUDA_TRY(cudaGetDevice(&dev));
        if (dev < 0 || dev >= 64 || !g_rader_ready[dev])
            return set_error(S2DWC_ERROR_NOT_INIT, "the length-511 alpha tables are not built on device %d", dev);
        if (a.mode == CZT_ANA_ALPHA) return launch_pfa511<CZT_ANA_ALPHA>(a, s);
        if (a.mode == CZT_SYN_ALPHA) return launch_pfa511<CZT_SYN_ALPHA>(a, s);
    }
    if (g_pfa && g_pfa1023 && a.bl == 512 && 2 * a.bl - 1 == PFC_N && a.rows % a.bl == 0) {
        if (a.mode == CZT_ANA_ALPHA) return launch_pfa1023<CZT_ANA_ALPHA>(a, s);
        if (a.mode == CZT_SYN_ALPHA) return launch_pfa1023<CZT_SYN_ALPHA>(a, s);
    }
    if (g_pfa && a.bl == 2048 && 2 * a.bl - 1 == PFA_N && a.rows % a.bl == 0) {
        if (a.mode == CZT_ANA_ALPHA) return launch_pfa<CZT_ANA_ALPHA>(a, s);
        if (a.mode == CZT_SYN_ALPHA) return launch_pfa<CZT_SYN_ALPHA>(a, s);
    }
    if (g_pfa && a.bl == 1024 && 2 * a.bl - 1 == PFB_N && a.rows % a.bl == 0) {
        int dev = 0;
        S2DW_CUDA_TRY(cudaGetDevice(&dev));
        if (dev < 0 || dev >= 64 || !g_rader_ready[dev])
            return set_error(S2DWC_ERROR_NOT_INIT, "the length-2047 alpha tables are not built on device %d", dev);
        if (g_pfa2047_threads == 128) {
            if (a.mode == CZT_ANA_ALPHA) return launch_pfa2047<CZT_ANA_ALPHA, 128>(a, s);
            if (a.mode == CZT_SYN_ALPHA) return launch_pfa2047<CZT_SYN_ALPHA, 128>(a, s);
        } else {
            if (a.mode == CZT_ANA_ALPHA) return launch_pfa2047<CZT_ANA_ALPHA, 256>(a, s);
            if (a.mode == CZT_SYN_ALPHA) return launch_pfa2047<CZT_SYN_ALPHA, 256>(a, s);
        }
    }
    const int M = a.czt.M;
    if (M < 16 || M > 8192 || (M & (M - 1)))
        return set_error(S2DWC_ERROR_SIZE_INVALID, "transform size %d unsupported", M);
    if (a.rows % a.bl == 0 && g_fft_values != 0) {
        // Stages whose input row is contiguous: persistent kernel with the
        // next row prefetched (synthesis alpha 4% faster than one row per
        // CTA at bl = 1024).  The analysis alpha stage stays one row per
        // CTA: its row-strided input gathered by cp.async gave no gain over
        // 256-bit loads (the chirp-table loads from L2, not the input,
        // dominate its remaining memory stalls).
        if (g_alpha_prefetch && a.mode == CZT_SYN_ALPHA && ((uintptr_t)a.in_r & 15) == 0) {
            if (M == 2048 && g_large_2048) return launch_pf<CZT_SYN_ALPHA, 11>(a, s);
            if (M == 4096) return launch_pf<CZT_SYN_ALPHA, 12>(a, s);
            if (M == 8192) return launch_pf<CZT_SYN_ALPHA, 13>(a, s);
        }
        if (g_alpha_prefetch && a.mode == FFT_ANA_BETA && ((uintptr_t)a.in_c & 15) == 0) {
            if (M == 2048 && g_large_2048) return launch_pf<FFT_ANA_BETA, 11>(a, s);
            if (M == 4096) return launch_pf<FFT_ANA_BETA, 12>(a, s);
        }
        if (M == 2048 && g_large_2048) return launch_large<11>(a, s);
        if (M == 4096) return launch_large<12>(a, s);
        if (M == 8192) return launch_large<13>(a, s);
    }
    if (g_fft_values == 16) return M <= 4096 ? launch_fft_mode<16, 256>(a, s) : launch_fft_mode<16, 512>(a, s);
    return M <= 4096 ? launch_fft_mode<8, 512>(a, s) : launch_fft_mode<8, 1024>(a, s);
}

void set_fft_values(int v) { g_fft_values = (v == 16) ? 16 : (v == 0 ? 0 : 8); }
void set_large_2048(bool on) { g_large_2048 = on; }

int launch_combine(const CombineArgs &a, cudaStream_t s)
{
    long long n = (long long)a.B * a.B, blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    combine_kernel<<<(int)blocks, 256, 0, s>>>(a);
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
