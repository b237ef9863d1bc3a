// Internal declarations shared by the host and device parts of libs2dw_cuda.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <exception>
#include <new>
#include <string>
#include <vector>

#include "../../include/s2dw_cuda.h"

namespace s2dw {

// ---------------------------------------------------------------------------
// Errors: every failing entry point records a code and a message.
// ---------------------------------------------------------------------------
int set_error(int code, const char *fmt, ...);

#define S2DW_CUDA_TRY(call)                                                              \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return ::s2dw::set_error(S2DWC_ERROR_CUDA, "%s failed: %s (%s:%d)", #call,   \
                                     cudaGetErrorString(e_), __FILE__, __LINE__);        \
    } while (0)

// No C++ exception may cross the C ABI (a Fortran or ctypes caller would be
// terminated): the body of every int-returning entry point runs inside
// S2DW_API_TRY ... S2DW_API_CATCH, which turns a failed host allocation into
// S2DWC_ERROR_MEM_ALLOC_FAIL and any other exception into
// S2DWC_ERROR_ARG_INVALID with its message.
#define S2DW_API_TRY try {
#define S2DW_API_CATCH                                                                        \
    }                                                                                         \
    catch (const std::bad_alloc &) {                                                          \
        return ::s2dw::set_error(S2DWC_ERROR_MEM_ALLOC_FAIL, "%s: host allocation failed",    \
                                 __func__);                                                   \
    }                                                                                         \
    catch (const std::exception &ex_) {                                                       \
        return ::s2dw::set_error(S2DWC_ERROR_ARG_INVALID, "%s: %s", __func__, ex_.what());    \
    }                                                                                         \
    catch (...) {                                                                             \
        return ::s2dw::set_error(S2DWC_ERROR_ARG_INVALID, "%s: unexpected exception", __func__); \
    }

// ---------------------------------------------------------------------------
// Host helpers restating the reference's scalar routines.
// ---------------------------------------------------------------------------
bool assimilate_int(double x, int *y);
int comp_jmax(int B, double alpha);
bool params_valid(int J, int B, double alpha, int N /* <0: absent */);
void band_limits(int jj, int B, double alpha, int *bl_hi, int *bl_lo);
double quad_weight(double theta, int B);

// Positive n set of the transform: n in [0, N) with N+n odd (the k_indicator
// test of s2dw_core_mod.f90:693 / :1146).  Returns its size NP (<= 4 for N<=8).
int positive_nset(int N, int *nq);

// ---------------------------------------------------------------------------
// Recurrence tables for d^l_{m'm}(pi/2), built on the host in long double.
//   l-walk (fixed m', m, stepping l):   e_{l+1} = -a_m(l) a_m'(l) e_l - e_{l-1},
//                                       d = Om_l(m) Om_l(m') e
//   m'-walk (fixed l, m, stepping m' down): e_{m'-1} = m b(l,m') e_{m'} - e_{m'+1},
//                                       d = Gam(l,m') e
// Start values are stored as mantissa (double in [1,2)) and binary exponent.
// All 2-D tables are [l*B + x] with zeros where x > l.
// ---------------------------------------------------------------------------
// Azimuthal band limits: N <= S2DW_NMAX (FP64 form; the split form N <= 8),
// so at most S2DW_NPMAX values n >= 0 with N + n odd.
constexpr int S2DW_NMAX = 16;
constexpr int S2DW_NPMAX = S2DW_NMAX / 2;
// Largest scale index J (scales j = 0..J): per-scale arrays passed to kernels
// by value are sized by it (J+1 entries, under 2.2 KB of kernel arguments).
constexpr int S2DW_JMAX = 127;

struct RecTables {
    int B = 0, HN = 8;
    std::vector<double> Om, Acoef;     // l-walk scale chains and coefficients
    std::vector<double> Stm;           // l-walk start E(l0,k)/Om_l0(k) mantissa
    std::vector<int32_t> Ste;          //   ... exponent
    std::vector<double> Gam, Bcoef;    // m'-walk chains and coefficients
    std::vector<double> Em;            // edge values E(l,m)=sqrt(C(2l,l+m))/2^l
    std::vector<int32_t> Ee;
    std::vector<double> H;             // d^l_{m'n}(pi/2), n < HN: [(l*HN+n)*B + m']
};
void build_rec_tables(int B, int hn, RecTables &t);  // H for n < hn

// ---------------------------------------------------------------------------
// Chirp-z (Bluestein) transform specification:
//   y[b] = sum_{k<K} x[k] exp(2 pi i s (k+k0)(b+b0)/L),  b < Bout,
// with k0, b0 integers or half-integers (passed doubled).
// ---------------------------------------------------------------------------
struct CztSpec {
    int K, Bout, L, s, k0x2, b0x2, M;
};
int czt_size(int K, int Bout);  // power of two M >= max(16, K+Bout-1)
void build_czt_tables(const CztSpec &c, std::vector<double2> &pre, std::vector<double2> &post,
                      std::vector<double2> &Hf);
// exp(i pi k / (4 bl)) for k < bl: the pre/post twiddle of the FFT beta modes.
void build_beta_twiddles(int bl, std::vector<double2> &tw);
// Two-level twiddle tables for a power-of-two FFT of size M:
// W_M^x = hi[x >> 6] * lo[x & 63], W_M = exp(-2 pi i / M).
void build_twiddles(int M, std::vector<double2> &hi, std::vector<double2> &lo);

// ---------------------------------------------------------------------------
// Device kernels (s2dw_kernels.cu)
// ---------------------------------------------------------------------------
// Transform modes.  CZT_* are chirp-z (Bluestein) transforms of any length;
// FFT_ANA_BETA / FFT_SYN_BETA are the beta transforms as one power-of-two FFT
// of length L = 2*bl (used when 2*bl is a power of two, bl >= 8): the analysis
// beta sum is a DCT-III of length L (cos rows) or, on the reversed input, a
// DST-III (i sin rows); the synthesis beta sum with its +-m' fold is the
// matching DCT-II / DST-II.  Each runs as one complex FFT of length L with a
// pre-twiddle, an even/odd reordering and a post-twiddle (Makhoul's
// algorithm, complex-linear, so complex rows need no real/imaginary split).
enum CztMode {
    CZT_ANA_BETA = 0,
    CZT_ANA_ALPHA = 1,
    CZT_SYN_ALPHA = 2,
    CZT_SYN_BETA = 3,
    FFT_ANA_BETA = 4,
    FFT_SYN_BETA = 5
};

struct CztDev {
    int M = 0;
    CztSpec spec{};
    double2 *pre = nullptr, *post = nullptr, *Hf = nullptr;
};

struct TwDev {
    int M = 0;
    double2 *hi = nullptr, *lo = nullptr;
};

// Tables of the plan use a padded row stride Bp = roundup(B, 32) so that
// 32-wide tiles never read past a row.
struct LwalkArgs {
    int B, Bp, N, NP, bl, blo;
    int nq[S2DW_NPMAX];
    const double *Acoef;  // [l*Bp + x]
    const double *Stm;    // [l0*B + k]
    const int32_t *Ste;
    const double *G;      // [((l-blo-1)*NP + q)*Gs + m'] = Om(l,m') d^l_{m'n_q} K_j(l) s(l,n_q)
    int Gs;               // roundup(bl, 32)
    const double2 *F;     // [l*Bp + m] = Om(l,m) flm(l,m)
    double2 *Tg;          // [g][m][m'] N x bl x bl
    const int2 *tiles;    // (p-tile, m-tile) per CTA, longest walks first
    int ntiles;
    // 0: Tg = T.  1: G holds the second real part b of S = eta (a + i b)
    // (a general complex Slm): Tg += T with the +n terms times -i and the
    // -n terms times +i (conj(S) for n >= 0, S for n < 0).
    int acc_imag;
};

struct MwalkArgs {
    int B, Bp, N, NP, bl, blo;
    int nq[S2DW_NPMAX];
    const double *Bcoef;  // [l*Bp + m']
    const double *Em;     // [l*B + m]
    const int32_t *Ee;
    const double *G;      // [((l-blo-1)*NP + q)*Gs + m'] = Gam(l,m') d^l_{m'n_q} c_j(l,n_q)
    int Gs;               // roundup(bl, 8)
    const double2 *V2f;   // [(q*bl + m)*Vs + m']
    int Vs;               // roundup(bl, 8)
    double2 *part;        // this scale's flm contribution [(l-blo-1)*bl + m], m <= l
    // the same tables transposed for the two-l-per-thread kernel:
    // GT[(m' (NP+1) + q) Ts + l - blo - 1], q < NP: G; q = NP: b(l, m');
    // rows m' < roundup(bl, 8), Ts = roundup(bl - blo - 1, 64), zero padded
    const double *GT;
    int Ts;
    int tile_l, tile_m;   // the plan's tile shape (mwalk_tile_l / mwalk_tile_m when it was built)
    const int2 *tiles;    // (l-tile, m-tile) per CTA, longest walks first
    int ntiles;
    // 0: part = result.  1: G holds the second real part b of S = eta (a + i b)
    // (a general complex Slm): part += i * result.
    int acc_imag;
};
// Tile lists of the contraction kernels for one scale, ordered by decreasing
// work so that the longest walks start first.
void build_lwalk_tiles(int bl, int blo, int ws, std::vector<int2> &t);
void build_mwalk_tiles(int bl, int blo, int wq, int tl, std::vector<int2> &t);
int lwalk_tile_m(int NP);  // m values per lwalk CTA tile
int mwalk_tile_m(int NP);  // m values per mwalk CTA tile
int mwalk_tile_l(int NP);  // l values per mwalk CTA tile: 64 for the kernel that reads GT, else 32
struct GsTArgs {
    int Bp, NP, bl, blo, Gs, Ts, rows;  // rows = roundup(bl, 8)
    const double *G, *Bcoef;
    double *out;
};
int launch_gsyn_t(const GsTArgs &a, cudaStream_t s);

// flm(l,m) = sum_j part_j(l,m) + Phi2(l) scoeff(l,m), the scale sum of
// s2dw_core_mod.f90:1228-1253 in scale order followed by :1258-1261.
struct CombineArgs {
    int B, J, bs;
    int bl[S2DW_JMAX + 1], blo[S2DW_JMAX + 1];
    long long off[S2DW_JMAX + 1];  // offset of part_j in `parts` (complex values)
    const double2 *parts;
    const double2 *scoeff;
    const double *Phi2;
    double2 *flm;
};

// Per-scale factor tables G (see LwalkArgs / MwalkArgs), built at
// set_tables time: out[((l-blo-1)*NP+q)*stride + x] = T[l*Bp+x] *
// H[(l*8+nq)*B+x] * kappa[l*NP+q] for x <= l, x < bl; zero elsewhere.
struct GprepArgs {
    int B, Bp, NP, bl, blo, stride, hn;  // hn: n rows of H
    int nq[S2DW_NPMAX];
    const double *T, *H, *kappa;
    double *out;
};
struct CztArgs {
    int mode, bl, N, NP, rows;
    int nq[S2DW_NPMAX];
    CztDev czt;
    TwDev tw;
    const double2 *in_c;   // complex input (Tg, Tb, V)
    const double *in_r;    // real input (wavelet coefficients)
    double2 *out_c;        // complex output (Tb, V, V2f)
    int out_stride;        // row stride of V2f (CZT_SYN_BETA)
    double *out_r;         // real output (wavelet coefficients)
    const double *wq;      // quadrature weights (2bl) for CZT_SYN_BETA
    double scale;          // (4 pi^2/N)/(2bl-1) for CZT_SYN_ALPHA
};

int launch_lwalk(const LwalkArgs &a, cudaStream_t s);
int launch_gprep(const GprepArgs &a, cudaStream_t s);
// F[l*Bp + m] = Om[l*Bp + m] * flm[l + B*m] for m <= l < B, zero for m > l.
int launch_fprep(double2 *F, const double2 *flm, const double *Om, int B, int Bp, cudaStream_t s);
int launch_mwalk(const MwalkArgs &a, cudaStream_t s);
int launch_czt(const CztArgs &a, cudaStream_t s);
void set_fft_values(int v);  // FFT engine variant: 8 or 16 values per thread, 0 = general engine only
void set_large_2048(bool on);  // M = 2048 transforms on the one-row-per-CTA engines (default on)
void set_pfa(bool on);  // prime-factor alpha stages at bl = 2048 and 1024 (default on)
void set_pfa2047_threads(int n);  // threads per CTA of the length-2047 kernel (128 or 256)
void set_pfa1023(bool on);         // prime-factor alpha stages at bl = 512
void set_pfa511(bool on);          // prime-factor alpha stages at bl = 256
void set_pfa_small(bool on);       // prime-factor alpha stages at bl = 2, 4, 8, 16, 32, 128
// Builds, once per device, the constant table of the length-2047 alpha stages
// (the current device; synchronises).  Plan creation calls it, never a capture.
int pfa_prepare();
void set_alpha_prefetch(bool on);  // synthesis alpha / analysis beta stages: persistent kernel with prefetched input (default on)
void set_walk_variants(int lwalk, int mwalk);  // tile shape / occupancy variants of the contraction kernels
int launch_zero(double *p, long long n, cudaStream_t s);
int launch_scoeff_copy(double2 *scoeff, const double2 *flm, int B, int bs, cudaStream_t s);
int launch_scaling_add(double2 *flm, const double2 *scoeff, const double *Phi2, int B, int bs,
                       cudaStream_t s);
int launch_combine(const CombineArgs &a, cudaStream_t s);

// ---------------------------------------------------------------------------
// Split-precision analysis contraction (tcgen05 int8 digits, batches of maps)
// ---------------------------------------------------------------------------
// Start values below 2^S2DW_SCALE_EXP put a warp of l-walk chains in a scaled
// domain; values above 2^S2DW_RENORM_EXP there are scaled back down.
#define S2DW_SCALE_EXP (-600)
#define S2DW_RENORM_EXP 400

struct SplitArgs {
    int B, Bp, N, NP, bl, blo;
    int c0, nch, nmaps;        // first 32-row chunk of l stored in fdig, chunks, maps (<= 32)
    int nq[S2DW_NPMAX];
    const double *Acoef, *Om;  // [l*Bp + x]
    const double *Stm;         // [l0*B + k]
    const int32_t *Ste;
    const double *G;           // as LwalkArgs::G
    int Gs;
    int16_t *dexp;             // [(m*bl + m')*NP + q] exponent of max_l |v|
    const int32_t *fexp;       // [m*64 + col] exponent of the map column
    const uint8_t *fdig;       // [(m*nch + chunk)*5 + digit][2048] map digits
    double2 *Tg;               // [k][g][m][m'] per map
    const double2 *ph;         // [g*16 + n+N-1] = exp(i pi n g / N)
    const int2 *tiles;         // (m, chain tile)
    int ntiles;
    int *err;                  // set to 1 when a wait gave up
    unsigned long long wait_ns;  // bound on every pipeline wait (the plan's wait limit)
};

struct FdigArgs {
    int B, bl, blo, c0, nch, nmaps;
    const double2 *flm;        // nmaps maps of B*B, flm[l + B*m]
    int32_t *fexp;
    uint8_t *fdig;
};

// Synthesis counterpart: for one m, rows are 128 chains l (m'-walk of
// d^l_{m'm}), K runs over (m', q) with MC m' and NPQ (power of two >= NP)
// values of q per 32-byte K step, columns are (map, re/im).
struct SplitSynArgs {
    int B, Bp, N, NP, bl, blo;
    int nch, nmaps;            // 32-row K chunks per m (MC m' each), maps (<= 32)
    const double *Bcoef;       // [l*Bp + m']
    const double *Em;          // [l*B + m]
    const int32_t *Ee;
    const double *G;           // as MwalkArgs::G
    int Gs;
    int16_t *sexp;             // [m*bl + l] exponent of max over (m', q) of |v|
    const int32_t *vexp;       // [m*64 + col]
    const uint8_t *vdig;       // [(m*nch + chunk)*6 + digit][2048] map digits
    double2 *part;             // map k: part + k*pstride, [(l-blo-1)*bl + m]
    long long pstride;
    const int2 *tiles;         // (m, 128-row l tile)
    int ntiles;
    int *err;
    unsigned long long wait_ns;
};

struct VdigArgs {
    int bl, NP, nch, nmaps, Vs;
    const double2 *V2f;        // map k: V2f + k*vstride, [(q*bl + m)*Vs + m']
    long long vstride;
    int32_t *vexp;
    uint8_t *vdig;
};

int split_syn_mc(int NP);       // m' per K chunk
long long split_vdig_bytes(int bl, int nch);
int launch_split_syn_dexp(const SplitSynArgs &a, cudaStream_t s);
int launch_split_vdig(const VdigArgs &a, cudaStream_t s);
int launch_split_syn(const SplitSynArgs &a, cudaStream_t s);

int split_chains(int NP);       // m' per CTA
int split_maps_per_pass();      // maps per CTA
long long split_fdig_bytes(int bl, int nch);
int launch_split_dexp(const SplitArgs &a, cudaStream_t s);
int launch_split_fdig(const FdigArgs &a, cudaStream_t s);
int launch_split(const SplitArgs &a, cudaStream_t s);

// ---------------------------------------------------------------------------
// Moments of the wavelet coefficients per scale (s2dw_stats.cu)
// ---------------------------------------------------------------------------
constexpr int STAT_P = 64;  // blocks per (map, scale) in the reduction passes
struct StatArgs {
    int J, nmaps;
    long long wtot;            // doubles per map in the packed layout
    long long off[S2DW_JMAX + 2];  // scale offsets (J+2 entries)
    const double *wav;         // map k at wav + k*wtot
    const double *mask;        // packed layout of one map, or null
    double *part;              // nmaps*(J+1)*STAT_P*6 partial sums
    double *mean_nj;           // nmaps*(J+1)*2
    double *out;               // nmaps*(J+1)*6: mean, var, skew, kur, five, six
    int *flags;                // nmaps*(J+1): 1 zero variance, 2 fewer than two samples
};
int launch_stat_moments(const StatArgs &a, cudaStream_t s);

// Address on `device` (which must be current) of the static scratch array of
// s2dwc_plan_analysis_noalloc, looked up once per device.
int noalloc_scratch(int device, void **ptr);
// Drops the cached addresses (s2dwc_finalize): the next call looks them up again.
void noalloc_forget();

}  // namespace s2dw
