// Host-side (FP64 / long double) parts of libs2dw_cuda: error state, the
// reference's scalar helpers and kernel tables, and the tables that drive the
// device recurrences and chirp-z transforms.
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "s2dw_internal.h"

namespace s2dw {

// ---------------------------------------------------------------------------
// Error state
// ---------------------------------------------------------------------------
static thread_local char g_last_msg[512] = "";

int set_error(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_msg, sizeof(g_last_msg), fmt, ap);
    va_end(ap);
    return code;
}

// ---------------------------------------------------------------------------
// Scalar helpers (s2dw_core_mod.f90:1327-1450)
// ---------------------------------------------------------------------------
static const double kTolCeil = 1e-5;     // TOL_CEIL, s2dw_types_mod.f90:60
static const double kTolQuad = 1e-12;    // TOL_QUAD, :54
static const double kTolLimit = 1e-12;   // TOL_LIMIT, :57
static const double kTolAdmiss = (double)1e-12f;  // TOL_ADMISS is a default-real literal, :48

// s2dw_core_assimilate_int, s2dw_core_mod.f90:1398-1415
bool assimilate_int(double x, int *y)
{
    double f = std::floor(x), c = std::ceil(x);
    if (std::fabs(x - f) < kTolCeil) { *y = (int)f; return true; }
    if (std::fabs(x - c) < kTolCeil) { *y = (int)c; return true; }
    *y = 0;
    return false;
}

// s2dw_core_comp_Jmax, s2dw_core_mod.f90:1365-1376
int comp_jmax(int B, double alpha)
{
    double x = std::log((double)B) / std::log(alpha);
    int j;
    if (!assimilate_int(x, &j)) j = (int)std::ceil(x);
    return j;
}

// s2dw_core_params_valid, s2dw_core_mod.f90:1327-1345
bool params_valid(int J, int B, double alpha, int N)
{
    int jmax = comp_jmax(B, alpha);
    bool ok = !(J > jmax || J < 1);
    if (N >= 0 && N > B) ok = false;
    return ok;
}

// Per-scale band limits, s2dw_core_mod.f90:372-381.
void band_limits(int jj, int B, double alpha, int *bl_hi, int *bl_lo)
{
    double xh = B / std::pow(alpha, (double)(jj - 1));
    double xl = B / std::pow(alpha, (double)(jj + 1));
    int hi, lo;
    if (!assimilate_int(xh, &hi)) hi = (int)std::ceil(xh);
    if (hi > B) hi = B;
    if (!assimilate_int(xl, &lo)) lo = (int)std::floor(xl);
    if (lo < 0) lo = 0;
    *bl_hi = hi;
    *bl_lo = lo;
}

// quad_weights, s2dw_core_mod.f90:1436-1450 (Driscoll-Healy weights)
double quad_weight(double theta, int B)
{
    double w = 0.0;
    for (int k = 0; k < B; k++) w += std::sin((2.0 * k + 1.0) * theta) / (2.0 * k + 1.0);
    return (2.0 / (double)B) * std::sin(theta) * w;
}

int positive_nset(int N, int *nq)
{
    int np = 0;
    for (int n = 0; n < N; n++)
        if ((N + n) % 2) nq[np++] = n;
    return np;
}

// ---------------------------------------------------------------------------
// Kernel tables: s2dw_core_mod.f90:97-304 and the quadrature it uses
// ---------------------------------------------------------------------------

// Integrand K_Phi^2(k)/k, s2dw_core_mod.f90:182-199.
static double phi2_integrand(double k, int bw, double alpha)
{
    int lo;
    if (!assimilate_int((double)bw / alpha, &lo)) lo = (int)std::floor((double)bw / alpha);
    double t = 2.0 * ((k - lo) / (double)(bw - lo)) - 1.0;
    return std::exp(-2.0 / (1.0 - t * t)) / k;
}

// Simpson's rule by successive trapezoid refinement (the Numerical Recipes
// scheme of s2dw_core_mod.f90:1586-1621 and :1724-1759: stop after more than
// five refinements once successive estimates agree to TOL_QUAD, at most 40).
static int simpson(int bw, double alpha, double a, double b, double *out)
{
    double st = 0.0, os = 0.0, ost = 0.0;
    for (int j = 1; j <= 40; j++) {
        if (j == 1) {
            st = 0.5 * (b - a) * (phi2_integrand(a, bw, alpha) + phi2_integrand(b, bw, alpha));
        } else {
            int it = 1 << (j - 2);
            double del = (b - a) / (double)it, x = a + 0.5 * del, sum = 0.0;
            for (int i = 0; i < it; i++) { sum += phi2_integrand(x, bw, alpha); x += del; }
            st = 0.5 * (st + (b - a) * sum / (double)it);
        }
        double s = (4.0 * st - ost) / 3.0;
        if (j > 5 && (std::fabs(s - os) < kTolQuad * std::fabs(os) || (s == 0.0 && os == 0.0))) {
            *out = s;
            return S2DWC_OK;
        }
        os = s;
        ost = st;
    }
    *out = os;
    return S2DWC_ERROR_QUAD_STEP_EXCEED;
}

}  // namespace s2dw

using namespace s2dw;

extern "C" {

int s2dwc_assimilate_int(double x, int *y)
{
    S2DW_API_TRY
    int t = 0;
    bool ok = assimilate_int(x, &t);
    if (y) *y = t;
    return ok ? 1 : 0;
    S2DW_API_CATCH
}

int s2dwc_comp_jmax(int B, double alpha) { return comp_jmax(B, alpha); }

const char *s2dwc_last_error_message(void) { return g_last_msg; }

int s2dwc_band_limits(int jj, int B, double alpha, int *bl_hi, int *bl_lo)
{
    S2DW_API_TRY
    if (!bl_hi || !bl_lo) return set_error(S2DWC_ERROR_ARG_INVALID, "band_limits: null output");
    band_limits(jj, B, alpha, bl_hi, bl_lo);
    return S2DWC_OK;
    S2DW_API_CATCH
}

long long s2dwc_wav_scale_size(int jj, int B, int N, double alpha)
{
    int hi, lo;
    band_limits(jj, B, alpha, &hi, &lo);
    return (long long)(2 * hi - 1) * (2 * hi) * N;
}

// s2dw_core_init_kernels, s2dw_core_mod.f90:97-157.  The B*(J+2) integrals
// are independent and run in parallel; each is the reference's Simpson
// iteration, so the values match it.
int s2dwc_init_kernels(double *K_gamma, double *Phi2, int *bl_scoeff, int J, int B, double alpha)
{
    S2DW_API_TRY
    if (!K_gamma || !Phi2 || !bl_scoeff)
        return set_error(S2DWC_ERROR_ARG_INVALID, "init_kernels: null pointer");
    if (B < 1 || !(alpha > 1.0) || !params_valid(J, B, alpha, -1))
        return set_error(S2DWC_ERROR_SIZE_INVALID, "init_kernels: invalid sizes J=%d B=%d alpha=%g",
                         J, B, alpha);
    const int nj = J + 2;
    std::vector<double> phi2((size_t)nj * B);
    std::vector<int> bws(nj), lows(nj);
    std::vector<double> cphi(nj);
    int status = S2DWC_OK;
    for (int jj = 0; jj < nj; jj++) {
        double xb = B / std::pow(alpha, (double)(jj - 1));
        int bw, lo;
        if (!assimilate_int(xb, &bw)) bw = (int)std::ceil(xb);
        if (!assimilate_int((double)bw / alpha, &lo)) lo = (int)std::floor((double)bw / alpha);
        bws[jj] = bw;
        lows[jj] = lo;
        int st = simpson(bw, alpha, (double)lo + kTolLimit, (double)bw - kTolLimit, &cphi[jj]);
        if (st != S2DWC_OK) status = st;
    }
#pragma omp parallel for schedule(dynamic, 4) collapse(2) reduction(max : status)
    for (int jj = 0; jj < nj; jj++) {
        for (int el = 0; el < B; el++) {
            double v;
            if (el <= lows[jj]) {
                v = 1.0;
            } else if (el >= bws[jj]) {
                v = 0.0;
            } else {
                double s;
                int st = simpson(bws[jj], alpha, (double)el, (double)bws[jj] - kTolLimit, &s);
                if (st != S2DWC_OK) status = st;
                v = s / cphi[jj];
            }
            phi2[jj + (size_t)nj * el] = v;
        }
    }
    for (int el = 0; el < B; el++) {
        for (int jj = 1; jj < nj; jj++) {
            double d = phi2[(jj - 1) + (size_t)nj * el] - phi2[jj + (size_t)nj * el];
            K_gamma[(jj - 1) + (size_t)(J + 1) * el] = d < 0.0 ? 0.0 : std::sqrt(d);
        }
        Phi2[el] = phi2[(J + 1) + (size_t)nj * el];
    }
    *bl_scoeff = bws[J + 1];
    if (status != S2DWC_OK)
        return set_error(status, "init_kernels: quadrature did not converge in 40 refinements");
    return S2DWC_OK;
    S2DW_API_CATCH
}

// ln(n!) by the Lanczos series the reference uses (s2dw_core_mod.f90:1497-1544).
// Its constants are default-real (single precision) literals in the
// reference, so they are rounded to float here to give the same binomials.
static double lanczos_logfact(int n)
{
    static const float c[6] = {76.18009172947146f, -86.50532032941677f, 24.01409824083091f,
                               -1.231739572450155f, 0.1208650973866179e-2f, -0.5395239384953e-5f};
    double x = (double)n + 1.0, y = x, ser = (double)1.000000000190015f;
    double tmp = x + 5.5 - (x + 0.5) * std::log(x + 5.5);
    for (int k = 0; k < 6; k++) { y += 1.0; ser += (double)c[k] / y; }
    return -tmp + std::log((double)2.5066282746310005f * ser / x);
}

// s2dw_core_init_directionality, s2dw_core_mod.f90:219-250.
int s2dwc_init_directionality(double *Slm_, int B, int N)
{
    S2DW_API_TRY
    if (!Slm_) return set_error(S2DWC_ERROR_ARG_INVALID, "init_directionality: null pointer");
    if (N > B || N < 1 || B < 1)
        return set_error(S2DWC_ERROR_SIZE_INVALID, "init_directionality: invalid N=%d B=%d", N, B);
    std::complex<double> *S = reinterpret_cast<std::complex<double> *>(Slm_);
    std::fill(S, S + (size_t)B * N, std::complex<double>(0.0, 0.0));
    const std::complex<double> eta = ((N - 1) % 2 == 0) ? std::complex<double>(1, 0)
                                                        : std::complex<double>(0, 1);
    for (int el = 1; el < B; el++) {
        int mmax = std::min(el, N - 1);
        for (int m = 0; m <= mmax; m++) {
            if ((N + m) % 2 == 0) continue;  // betah = 0
            int g = std::min(N - 1, el - (((N + el) % 2) ? 0 : 1));
            int r = (g - m) / 2;
            double lb = lanczos_logfact(g) - lanczos_logfact(r) - lanczos_logfact(g - r);
            int binom = (int)std::floor(0.5 + std::exp(lb));
            S[el + (size_t)B * m] = std::sqrt((double)binom / std::pow(2.0, (double)g)) * eta;
        }
    }
    return S2DWC_OK;
    S2DW_API_CATCH
}

// s2dw_core_admiss, s2dw_core_mod.f90:285-304.
int s2dwc_admiss(double *admiss, const double *K_gamma, const double *Phi2, int B, int J, int *pass)
{
    S2DW_API_TRY
    if (!admiss || !K_gamma || !Phi2)
        return set_error(S2DWC_ERROR_ARG_INVALID, "admiss: null pointer");
    int ok = 1;
    for (int el = 0; el < B; el++) {
        double a = Phi2[el];
        for (int jj = 0; jj <= J; jj++) {
            double k = K_gamma[jj + (size_t)(J + 1) * el];
            a += k * k;
        }
        admiss[el] = a;
        if (std::fabs(a - 1.0) > kTolAdmiss) ok = 0;
    }
    if (pass) *pass = ok;
    return S2DWC_OK;
    S2DW_API_CATCH
}

}  // extern "C"

namespace s2dw {

// ---------------------------------------------------------------------------
// Recurrence tables (long double on the host, stored as double)
// ---------------------------------------------------------------------------
typedef long double ld;

static void split_mant_exp(ld v, double *mant, int32_t *ex)
{
    if (v == 0.0L) { *mant = 0.0; *ex = 0; return; }
    int e;
    ld f = frexpl(v, &e);  // v = f 2^e, |f| in [0.5,1)
    *mant = (double)(2.0L * f);
    *ex = e - 1;
}

void build_rec_tables(int B, int hn, RecTables &t)
{
    t.B = B;
    t.HN = hn;
    const size_t BB = (size_t)B * B;
    t.Om.assign(BB, 0.0);
    t.Acoef.assign(BB, 0.0);
    t.Stm.assign(BB, 0.0);
    t.Ste.assign(BB, 0);
    t.Gam.assign(BB, 0.0);
    t.Bcoef.assign(BB, 0.0);
    t.Em.assign(BB, 0.0);
    t.Ee.assign(BB, 0);
    t.H.assign(BB * hn, 0.0);

    // Edge values E(l,k) = sqrt(C(2l,l+k))/2^l = |d^l_{l,k}(pi/2)| by exact
    // products (E(l,0)^2 = prod (2i-1)/(2i); E(l,k)/E(l,k-1) = sqrt((l-k+1)/(l+k))).
    std::vector<ld> E(BB, 0.0L);
    {
        ld e0 = 1.0L;
        for (int l = 0; l < B; l++) {
            if (l > 0) e0 *= sqrtl((ld)(2 * l - 1) / (ld)(2 * l));
            ld e = e0;
            E[(size_t)l * B] = e;
            for (int k = 1; k <= l; k++) {
                e *= sqrtl((ld)(l - k + 1) / (ld)(l + k));
                E[(size_t)l * B + k] = e;
            }
        }
    }
    auto u_of = [](int l, int x) -> ld {  // coefficient of d^l in the l recurrence
        return sqrtl((ld)(2 * l + 1) / (ld)l) * (ld)x / sqrtl((ld)(l + 1) * (l + 1) - (ld)x * x);
    };
    auto v_of = [](int l, int x) -> ld {  // coefficient of d^{l-1}
        return sqrtl((ld)(l + 1) / (ld)l) * sqrtl((ld)l * l - (ld)x * x) /
               sqrtl((ld)(l + 1) * (l + 1) - (ld)x * x);
    };

    // l-walk chains Om_l(x): Om_x = Om_{x+1} = 1, Om_{l+1} = v_x(l) Om_{l-1};
    // a_x(l) = u_x(l) Om_l(x)/Om_{l+1}(x).
#pragma omp parallel for schedule(dynamic, 8)
    for (int x = 0; x < B; x++) {
        std::vector<ld> om(B + 2, 0.0L);
        om[x] = 1.0L;
        om[x + 1] = 1.0L;
        for (int l = x + 1; l < B; l++) om[l + 1] = v_of(l, x) * om[l - 1];
        for (int l = x; l < B; l++) {
            t.Om[(size_t)l * B + x] = (double)om[l];
            ld a = (l == 0) ? 0.0L : u_of(l, x) * om[l] / om[l + 1];
            t.Acoef[(size_t)l * B + x] = (double)a;
        }
    }
    // l-walk start: pair with larger index l0 and smaller k starts at
    // E(l0,k)/Om_l0(k) (the larger index has Om = 1); the sign is applied on
    // the device.
    for (int l0 = 0; l0 < B; l0++)
        for (int k = 0; k <= l0; k++) {
            ld om = (ld)t.Om[(size_t)l0 * B + k];
            split_mant_exp(E[(size_t)l0 * B + k] / om, &t.Stm[(size_t)l0 * B + k],
                           &t.Ste[(size_t)l0 * B + k]);
            split_mant_exp(E[(size_t)l0 * B + k], &t.Em[(size_t)l0 * B + k],
                           &t.Ee[(size_t)l0 * B + k]);
        }

    // m'-walk chains: gamma(l,m') = sqrt((l+m')(l-m'+1)); Gam(l,l)=Gam(l,l-1)=1,
    // Gam(l,m'-1) = Gam(l,m'+1) gamma(l,m'+1)/gamma(l,m');
    // b(l,m') = 2 Gam(l,m') / (gamma(l,m') Gam(l,m'-1)).
#pragma omp parallel for schedule(dynamic, 8)
    for (int l = 0; l < B; l++) {
        std::vector<ld> G(l + 2, 0.0L);
        auto gam = [l](int mp) { return sqrtl((ld)(l + mp) * (ld)(l - mp + 1)); };
        G[l] = 1.0L;
        if (l >= 1) G[l - 1] = 1.0L;
        for (int mp = l - 1; mp >= 1; mp--) G[mp - 1] = G[mp + 1] * gam(mp + 1) / gam(mp);
        for (int mp = 0; mp <= l; mp++) {
            t.Gam[(size_t)l * B + mp] = (double)G[mp];
            if (mp >= 1) t.Bcoef[(size_t)l * B + mp] = (double)(2.0L * G[mp] / (gam(mp) * G[mp - 1]));
        }
    }

    // H(l,m',n) = d^l_{m'n}(pi/2), n < hn, by the l recurrence in long double.
#pragma omp parallel for schedule(dynamic, 8)
    for (int mp = 0; mp < B; mp++) {
        for (int n = 0; n < hn && n < B; n++) {
            int l0 = mp > n ? mp : n;
            ld d = (mp >= n) ? (((l0 - n) & 1) ? -E[(size_t)l0 * B + n] : E[(size_t)l0 * B + n])
                             : E[(size_t)l0 * B + mp];
            ld dp = 0.0L;
            for (int l = l0; l < B; l++) {
                t.H[((size_t)l * hn + n) * B + mp] = (double)d;
                ld dn;
                if (l == 0) dn = 0.0L;
                else dn = -u_of(l, mp) * u_of(l, n) * d - v_of(l, mp) * v_of(l, n) * dp;
                dp = d;
                d = dn;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Chirp-z tables
// ---------------------------------------------------------------------------
int czt_size(int K, int Bout)
{
    int need = K + Bout - 1, M = 16;
    while (M < need) M *= 2;
    return M;
}

// Forward FFT (sign -1) of size M (power of two) in long double.
static void fft_ld(std::vector<std::complex<ld>> &a)
{
    const size_t n = a.size();
    for (size_t i = 1, j = 0; i < n; i++) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    const ld pi = 3.141592653589793238462643383279502884L;
    for (size_t len = 2; len <= n; len <<= 1) {
        for (size_t i = 0; i < n; i += len)
            for (size_t k = 0; k < len / 2; k++) {
                ld ang = -2.0L * pi * (ld)k / (ld)len;
                std::complex<ld> w(cosl(ang), sinl(ang));
                std::complex<ld> u = a[i + k], v = a[i + k + len / 2] * w;
                a[i + k] = u + v;
                a[i + k + len / 2] = u - v;
            }
    }
}

// exp(i pi s z^2 / L) for z = Z2/2 with exact reduction of the phase.
static std::complex<ld> chirp(long long Z2, int L, int s)
{
    const ld pi = 3.141592653589793238462643383279502884L;
    long long q = (Z2 * Z2) % (8LL * L);  // phase = pi s (Z2^2 mod 8L) / (4L)
    ld ang = pi * (ld)s * (ld)q / (ld)(4LL * L);
    return std::complex<ld>(cosl(ang), sinl(ang));
}

void build_czt_tables(const CztSpec &c, std::vector<double2> &pre, std::vector<double2> &post,
                      std::vector<double2> &Hf)
{
    pre.resize(c.K);
    post.resize(c.Bout);
    for (int k = 0; k < c.K; k++) {
        auto v = chirp(2LL * k + c.k0x2, c.L, c.s);
        pre[k] = make_double2((double)v.real(), (double)v.imag());
    }
    for (int b = 0; b < c.Bout; b++) {
        auto v = chirp(2LL * b + c.b0x2, c.L, c.s);
        post[b] = make_double2((double)v.real(), (double)v.imag());
    }
    std::vector<std::complex<ld>> h(c.M, std::complex<ld>(0, 0));
    const long long cx2 = (long long)c.b0x2 - c.k0x2;
    for (int d = -(c.K - 1); d <= c.Bout - 1; d++) {
        auto v = std::conj(chirp(2LL * d + cx2, c.L, c.s));
        h[((d % c.M) + c.M) % c.M] = v;
    }
    fft_ld(h);
    Hf.resize(c.M);
    for (int k = 0; k < c.M; k++)
        Hf[k] = make_double2((double)(h[k].real() / c.M), (double)(h[k].imag() / c.M));
}

void build_beta_twiddles(int bl, std::vector<double2> &tw)
{
    const ld pi = 3.141592653589793238462643383279502884L;
    tw.resize(bl);
    for (int k = 0; k < bl; k++) {
        ld a = pi * (ld)k / (ld)(4LL * bl);
        tw[k] = make_double2((double)cosl(a), (double)sinl(a));
    }
}

void build_twiddles(int M, std::vector<double2> &hi, std::vector<double2> &lo)
{
    const ld pi = 3.141592653589793238462643383279502884L;
    int nhi = (M + 63) / 64;
    hi.resize(nhi);
    lo.resize(64);
    for (int i = 0; i < nhi; i++) {
        ld a = -2.0L * pi * (ld)(64LL * i) / (ld)M;
        hi[i] = make_double2((double)cosl(a), (double)sinl(a));
    }
    for (int i = 0; i < 64; i++) {
        ld a = -2.0L * pi * (ld)i / (ld)M;
        lo[i] = make_double2((double)cosl(a), (double)sinl(a));
    }
}

}  // namespace s2dw
