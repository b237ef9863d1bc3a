/*
 * s2dw_oracle.c -- CPU restatement of the S2DW v1.1 hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: it restates,
 * loop by loop, the reference Fortran routines that the CUDA library
 * replaces, so that tests can compare the GPU results with the reference's
 * algorithm on the same inputs.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it.  The product library never links
 * or calls it.
 *
 * Parity status: the reference is Fortran 90 + FFTW and no Fortran compiler
 * or FFTW exists on this machine, so the reference itself cannot be run and
 * it ships no golden vectors.  Parity of this restatement is therefore
 * "parity unpinned" by reference outputs; it is pinned instead by
 * known-answer tests (closed-form and high-precision Wigner-d values,
 * orthogonality, admissibility to 1e-12, and analysis->synthesis
 * reconstruction, which is the reference's own self-test criterion).
 *
 * Array conventions follow the Fortran column-major layouts exactly:
 *   flm(0:B-1,0:B-1)            -> flm[l + B*m]
 *   K_gamma(0:J,0:B-1)          -> K[j + (J+1)*l]
 *   Slm(0:B-1,0:N-1)            -> S[l + B*n]
 *   wav(0:J,0:2B-2,0:2B-1,0:N-1)-> wav[j + (J+1)*(a + (2B-1)*(b + 2B*g))]
 *   wavdyn(j)%coeff(0:2bl-2,0:2bl-1,0:N-1) -> c[a + (2bl-1)*(b + 2bl*g)]
 *   scoeff(0:bs-1,0:bs-1)       -> sc[l + bs*m]
 *   dl(-l:l,-l:l)               -> dl[(i+l) + (2l+1)*(k+l)]
 *
 * Citations are to files of the reference project (src/mod/...).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex dcx;

#define ORC_PI 3.141592653589793238462643383279502884197
#define ORC_PION2 1.570796326794896619231321691639751442099
/* s2dw_types_mod.f90:48-60.  TOL_ADMISS/TOL_ZERO are single-precision
 * literals in the reference (1e-12 without a d exponent). */
#define ORC_TOL_ADMISS ((double)1e-12f)
#define ORC_TOL_QUAD 1e-12
#define ORC_TOL_LIMIT 1e-12
#define ORC_TOL_CEIL 1e-5

/* error codes, s2dw_error_mod.f90:37-52 */
enum { ORC_OK = 0, ORC_ERR_MEM = 4, ORC_ERR_ARTH = 5, ORC_ERR_SIZE = 8,
       ORC_ERR_QUAD = 12, ORC_ERR_ADMISS = 13 };

/* ------------------------------------------------------------------ */
/* Helpers: s2dw_core_mod.f90:1327-1450                                */
/* ------------------------------------------------------------------ */

/* s2dw_core_assimilate_int, s2dw_core_mod.f90:1398-1415 */
int orc_assimilate_int(double x, int *y)
{
    if (fabs(x - floor(x)) < ORC_TOL_CEIL) { *y = (int)floor(x); return 1; }
    if (fabs(x - ceil(x)) < ORC_TOL_CEIL) { *y = (int)ceil(x); return 1; }
    *y = 0;
    return 0;
}

/* s2dw_core_comp_Jmax, s2dw_core_mod.f90:1365-1376 */
int orc_comp_jmax(int B, double alpha)
{
    int j;
    double x = log((double)B) / log(alpha);
    if (!orc_assimilate_int(x, &j)) j = (int)ceil(x);
    return j;
}

/* s2dw_core_params_valid, s2dw_core_mod.f90:1327-1345 (N<0: absent) */
int orc_params_valid(int J, int B, double alpha, int N)
{
    int jmax = orc_comp_jmax(B, alpha);
    int valid = 1;
    if (J > jmax || J < 1) valid = 0;
    if (N >= 0 && N > B) valid = 0;
    return valid;
}

/* Band limits of scale jj: s2dw_core_mod.f90:372-381 (repeated in every
 * transform routine). */
void orc_band_limits(int jj, int B, double alpha, int *bl_hi, int *bl_lo)
{
    int hi, lo;
    double xh = B / pow(alpha, (double)(jj - 1));
    double xl = B / pow(alpha, (double)(jj + 1));
    if (orc_assimilate_int(xh, &hi)) hi = hi < B ? hi : B;
    else { hi = (int)ceil(xh); hi = hi < B ? hi : B; }
    if (orc_assimilate_int(xl, &lo)) lo = lo > 0 ? lo : 0;
    else { lo = (int)floor(xl); lo = lo > 0 ? lo : 0; }
    *bl_hi = hi;
    *bl_lo = lo;
}

/* quad_weights, s2dw_core_mod.f90:1436-1450 */
double orc_quad_weights(double theta, int B)
{
    double w = 0.0;
    for (int k = 0; k <= B - 1; k++)
        w = w + sin((2.0 * k + 1.0) * theta) / (2.0 * k + 1.0);
    return (2.0 / (double)B) * sin(theta) * w;
}

/* logfact (Lanczos), s2dw_core_mod.f90:1497-1544.  The reference writes
 * the constants and 5.5/0.5/1.0 as default-real literals, which gfortran
 * rounds to single precision; that rounding is kept here. */
static double orc_logfact(int n)
{
    const double c[6] = {(double)76.18009172947146f, (double)-86.50532032941677f,
                         (double)24.01409824083091f, (double)-1.231739572450155f,
                         (double)0.1208650973866179e-2f, (double)-0.5395239384953e-5f};
    double x = (double)n + 1.0;
    double temp = x + 5.5 - (x + 0.5) * log(x + 5.5);
    double sum = (double)1.000000000190015f;
    double y = x;
    for (int k = 0; k < 6; k++) { y = y + 1.0; sum = sum + c[k] / y; }
    return -temp + log((double)2.5066282746310005f * sum / x);
}

/* binomial, s2dw_core_mod.f90:1470-1478 */
static int orc_binomial(int n, int r)
{
    return (int)floor(0.5 + exp(orc_logfact(n) - orc_logfact(r) - orc_logfact(n - r)));
}

/* ------------------------------------------------------------------ */
/* Kernel tables: s2dw_core_mod.f90:97-304, 1586-1759                  */
/* ------------------------------------------------------------------ */

/* s2dw_core_phi2_integrand, s2dw_core_mod.f90:182-199 */
static double orc_phi2_integrand(double k, int bw, double alpha)
{
    int bw_lo;
    if (!orc_assimilate_int((double)bw / alpha, &bw_lo)) bw_lo = (int)floor((double)bw / alpha);
    double t = 2.0 * ((k - bw_lo) / (double)(bw - bw_lo)) - 1.0;
    return exp(-2.0 / (1.0 - t * t)) / k;
}

/* trapzd, s2dw_core_mod.f90:1586-1621 */
static void orc_trapzd(int bw, double alpha, double a, double b, double *s, int n)
{
    if (n == 1) {
        *s = 0.5 * (b - a) * (orc_phi2_integrand(a, bw, alpha) + orc_phi2_integrand(b, bw, alpha));
    } else {
        int it = 1 << (n - 2);
        double del = (b - a) / (double)it;
        double x = a + 0.5 * del;
        double fsum = 0.0;
        for (int j = 1; j <= it; j++) { fsum = fsum + orc_phi2_integrand(x, bw, alpha); x = x + del; }
        *s = 0.5 * (*s + (b - a) * fsum / (double)it);
    }
}

/* qsimp, s2dw_core_mod.f90:1724-1759 (JMAX=40) */
static int orc_qsimp(int bw, double alpha, double a, double b, double *integral)
{
    double os = 0.0, ost = 0.0, st = 0.0;
    for (int j = 1; j <= 40; j++) {
        orc_trapzd(bw, alpha, a, b, &st, j);
        *integral = (4.0 * st - ost) / 3.0;
        if (j > 5) {
            if (fabs(*integral - os) < ORC_TOL_QUAD * fabs(os) || (*integral == 0.0 && os == 0.0))
                return ORC_OK;
        }
        os = *integral;
        ost = st;
    }
    return ORC_ERR_QUAD;
}

/* s2dw_core_init_kernels, s2dw_core_mod.f90:97-157 */
int orc_init_kernels(double *K_gamma, double *Phi2, int *bl_scoeff, int J, int B, double alpha)
{
    if (!orc_params_valid(J, B, alpha, -1)) return ORC_ERR_SIZE;
    double *phi2_all = (double *)malloc(sizeof(double) * (size_t)(J + 2) * (size_t)B);
    if (!phi2_all) return ORC_ERR_MEM;
    int bw = 0, status = ORC_OK;
#define PHI2(jj, el) phi2_all[(jj) + (size_t)(J + 2) * (el)]
    for (int jj = 0; jj <= J + 1; jj++) {
        double xb = B / pow(alpha, (double)(jj - 1));
        int el_lo;
        if (!orc_assimilate_int(xb, &bw)) bw = (int)ceil(xb);
        if (!orc_assimilate_int((double)bw / alpha, &el_lo)) el_lo = (int)floor((double)bw / alpha);
        double c_phi;
        int st = orc_qsimp(bw, alpha, (double)el_lo + ORC_TOL_LIMIT, (double)bw - ORC_TOL_LIMIT, &c_phi);
        if (st != ORC_OK) status = st;
        for (int el = 0; el <= B - 1; el++) {
            if (el <= el_lo) {
                PHI2(jj, el) = 1.0;
            } else if (el >= bw) {
                PHI2(jj, el) = 0.0;
            } else {
                double v;
                st = orc_qsimp(bw, alpha, (double)el, (double)bw - ORC_TOL_LIMIT, &v);
                if (st != ORC_OK) status = st;
                PHI2(jj, el) = v / c_phi;
            }
            if (jj >= 1) {
                double diff = PHI2(jj - 1, el) - PHI2(jj, el);
                K_gamma[(jj - 1) + (size_t)(J + 1) * el] = diff < 0.0 ? 0.0 : sqrt(diff);
            }
        }
    }
    for (int el = 0; el < B; el++) Phi2[el] = PHI2(J + 1, el);
#undef PHI2
    *bl_scoeff = bw;
    free(phi2_all);
    return status;
}

/* s2dw_core_init_directionality, s2dw_core_mod.f90:219-250 */
int orc_init_directionality(dcx *Slm, int B, int N)
{
    if (N > B) return ORC_ERR_SIZE;
    for (size_t i = 0; i < (size_t)B * N; i++) Slm[i] = 0.0;
    for (int el = 1; el <= B - 1; el++) {
        int mmax = el < N - 1 ? el : N - 1;
        for (int m = 0; m <= mmax; m++) {
            int betah = (1 - (((N + m) % 2) ? -1 : 1)) / 2;
            if (betah > 0) {
                int g = el - (1 + (((N + el) % 2) ? -1 : 1)) / 2;
                if (N - 1 < g) g = N - 1;
                int binom = orc_binomial(g, (g - m) / 2);
                dcx eta = ((N - 1) % 2 == 0) ? 1.0 : I;
                Slm[el + (size_t)B * m] = sqrt((double)binom / pow(2.0, (double)g)) * eta;
            }
        }
    }
    return ORC_OK;
}

/* s2dw_core_admiss, s2dw_core_mod.f90:285-304 */
int orc_admiss(double *admiss, const double *K_gamma, const double *Phi2, int B, int J)
{
    int pass = 1;
    for (int el = 0; el < B; el++) {
        double a = Phi2[el];
        for (int jj = 0; jj <= J; jj++) {
            double k = K_gamma[jj + (size_t)(J + 1) * el];
            a = a + k * k;
        }
        admiss[el] = a;
        if (fabs(a - 1.0) > ORC_TOL_ADMISS) pass = 0;
    }
    return pass;
}

/* ------------------------------------------------------------------ */
/* Wigner d plane: s2dw_dl_mod.f90:56-304 (Turok & Bucher operator)   */
/* ------------------------------------------------------------------ */

#define DL(i, k) dl[((i) + l) + (size_t)(2 * l + 1) * ((k) + l)]

/* s2dw_dl_beta_operator_core, s2dw_dl_mod.f90:92-238 */
static void orc_dl_core(double *dl, double beta, int l)
{
    if (fabs(beta) < 1e-5) {
        for (size_t i = 0; i < (size_t)(2 * l + 1) * (2 * l + 1); i++) dl[i] = 0.0;
        for (int i = -l; i <= l; i++) DL(i, i) = 1.0;
        return;
    }
    int lp1 = l + 1, n = 2 * l + 1;
    double *cp = (double *)malloc(sizeof(double) * (n + 1));
    double *cpi = (double *)malloc(sizeof(double) * (n + 1));
    double *cp2 = (double *)malloc(sizeof(double) * (n + 1));
    double *lfr = (double *)malloc(sizeof(double) * (n + 1));
    double *sgn = (double *)malloc(sizeof(double) * (n + 1));
    double *lren = (double *)malloc(sizeof(double) * (n + 1));
    const double big_const = 1.0e150;
    double ang = beta, c = cos(ang), s = sin(ang), si = 1.0 / s, t = tan(-ang / 2.0);
    double c2 = cos(ang / 2.0), omc = 1.0 - c;
    for (int i = 1; i <= n; i++) lren[i] = 0.0;
    /* first row, :140-148 */
    lfr[1] = (2.0 * (double)l) * log(fabs(c2));
    sgn[1] = 1.0;
    for (int i = 2; i <= n; i++) {
        int m = l + 1 - i;
        double ratio = sqrt((double)(l + m + 1) / (double)(l - m));
        lfr[i] = lfr[i - 1] + log(ratio) + log(fabs(t));
        sgn[i] = sgn[i - 1] * t / fabs(t);
    }
    double big = big_const, lbig = log(big), bigi = 1.0 / big_const;
    double xllp1 = (double)(l * (l + 1));
    /* :158-167 */
    for (int m = 1; m <= l; m++) {
        double xm = (double)(l - m);
        cpi[m] = 2.0 / sqrt(xllp1 - xm * (xm + 1));
        cp[m] = 1.0 / cpi[m];
    }
    for (int m = 2; m <= l; m++) cp2[m] = cpi[m] * cp[m - 1];
    DL(1 - lp1, 1 - lp1) = 1.0;
    DL(2 * l + 1 - lp1, 1 - lp1) = 1.0;
    /* recurrence down to the diagonals, :171-190 */
    for (int index = 2; index <= l + 1; index++) {
        DL(index - lp1, 1 - lp1) = 1.0;
        double lambda = ((double)(l + 1) * omc - (double)index + c) * si;
        DL(index - lp1, 2 - lp1) = lambda * DL(index - lp1, 1 - lp1) * cpi[1];
        if (index > 2) {
            for (int m = 2; m <= index - 1; m++) {
                lambda = ((double)(l + 1) * omc - (double)index + (double)m * c) / s;
                DL(index - lp1, m + 1 - lp1) =
                    lambda * cpi[m] * DL(index - lp1, m - lp1) - cp2[m] * DL(index - lp1, m - 1 - lp1);
                if (DL(index - lp1, m + 1 - lp1) > big) {
                    lren[index] = lren[index] - lbig;
                    for (int im = 1; im <= m + 1; im++) DL(index - lp1, im - lp1) *= bigi;
                }
            }
        }
    }
    /* other half of the triangle, :194-213 */
    for (int index = l + 2; index <= 2 * l; index++) {
        DL(index - lp1, 1 - lp1) = 1.0;
        double lambda = ((double)(l + 1) * omc - (double)index + c) / s;
        DL(index - lp1, 2 - lp1) = lambda * DL(index - lp1, 1 - lp1) * cpi[1];
        if (index < 2 * l) {
            for (int m = 2; m <= 2 * l - index + 1; m++) {
                lambda = ((double)(l + 1) * omc - (double)index + (double)m * c) / s;
                DL(index - lp1, m + 1 - lp1) =
                    lambda * cpi[m] * DL(index - lp1, m - lp1) - cp2[m] * DL(index - lp1, m - 1 - lp1);
                if (DL(index - lp1, m + 1 - lp1) > big) {
                    for (int im = 1; im <= m + 1; im++) DL(index - lp1, im - lp1) *= bigi;
                    lren[index] = lren[index] - lbig;
                }
            }
        }
    }
    /* renormalise, :215-227 */
    for (int i = 1; i <= l + 1; i++) {
        double renorm = sgn[i] * exp(lfr[i] - lren[i]);
        for (int j = 1; j <= i; j++) DL(i - lp1, j - lp1) *= renorm;
    }
    for (int i = l + 2; i <= 2 * l + 1; i++) {
        double renorm = sgn[i] * exp(lfr[i] - lren[i]);
        for (int j = 1; j <= 2 * l + 2 - i; j++) DL(i - lp1, j - lp1) *= renorm;
    }
    free(cp); free(cpi); free(cp2); free(lfr); free(sgn); free(lren);
}

/* s2dw_dl_beta_operator_fill, s2dw_dl_mod.f90:258-304 */
static void orc_dl_fill(double *dl, int l)
{
    int lp1 = l + 1;
    for (int i = 1; i <= l; i++)
        for (int j = l + 1; j <= 2 * l + 1 - i; j++)
            DL(2 * l + 2 - i - lp1, 2 * l + 2 - j - lp1) = DL(j - lp1, i - lp1);
    for (int i = 1; i <= l + 1; i++) {
        int sg = -1;
        for (int j = i + 1; j <= l + 1; j++) {
            DL(i - lp1, j - lp1) = DL(j - lp1, i - lp1) * sg;
            sg = -sg;
        }
    }
    for (int i = l + 2; i <= 2 * l + 1; i++) {
        int sg = ((i + 1) % 2) ? -1 : 1;
        for (int j = 1; j <= 2 * l + 2 - i; j++) {
            DL(j - lp1, i - lp1) = DL(i - lp1, j - lp1) * sg;
            sg = -sg;
        }
        for (int j = i; j <= 2 * l + 1; j++)
            DL(j - lp1, i - lp1) = DL(2 * l + 2 - i - lp1, 2 * l + 2 - j - lp1);
    }
    for (int i = l + 2; i <= 2 * l + 1; i++)
        for (int j = 2 * l + 3 - i; j <= i - 1; j++)
            DL(j - lp1, i - lp1) = DL(2 * l + 2 - i - lp1, 2 * l + 2 - j - lp1);
}
#undef DL

/* s2dw_dl_beta_operator, s2dw_dl_mod.f90:56-68.  dl holds (2l+1)^2 values,
 * dl(i,k) at (i+l) + (2l+1)*(k+l). */
void orc_dl_beta_operator(double *dl, double beta, int l)
{
    orc_dl_core(dl, beta, l);
    orc_dl_fill(dl, l);
}

/* DIAGNOSTIC, not the reference's algorithm: the plane d^l(pi/2) from the
 * three-term recurrence in the second index at fixed first index a,
 *   sqrt((l+b)(l-b+1)) d_{a,b-1} + sqrt((l-b)(l+b+1)) d_{a,b+1} = -2a d_{a,b},
 * walked in long double from the closed-form edge d^l_{a,l} = sqrt(C(2l,l+a))/2^l
 * (the edge values by exact ratios from 2^-l) down to b = 0, then
 * d^l_{a,-b} = (-1)^(l+a) d^l_{a,b}.  Walking inward from the edge follows the
 * dominant solution, so the planes stay within ~1e-17 of 50-digit values up
 * to l = 2047, where the reference's Turok-Bucher planes reach 1.4e-13.
 * Selected with orc_set_dl_method(1) to separate, in a comparison at large l,
 * the reference algorithm's own d-plane error from the rest. */
static int orc_dl_method = 0;
void orc_set_dl_method(int m) { orc_dl_method = m; }

void orc_dl_edge_ld(double *dl, int l)
{
    const size_t w = (size_t)(2 * l + 1);
    long double *r = (long double *)malloc(sizeof(long double) * (size_t)(2 * l + 3));
    long double *E = (long double *)malloc(sizeof(long double) * (size_t)(2 * l + 1));
    if (!r || !E) { free(r); free(E); return; }
    for (int b = -l; b <= l + 1; b++) r[b + l] = sqrtl((long double)(l + b) * (long double)(l - b + 1));
    E[2 * l] = ldexpl(1.0L, -l);  /* a = l: sqrt(C(2l,2l)) / 2^l */
    for (int a = l; a > -l; a--)  /* C(2l,l+a-1) = C(2l,l+a) (l+a)/(l-a+1) */
        E[a - 1 + l] = E[a + l] * sqrtl((long double)(l + a) / (long double)(l - a + 1));
    for (int a = -l; a <= l; a++) {
        long double dn = 0.0L, d = E[a + l];
        dl[(size_t)(a + l) + w * (size_t)(2 * l)] = (double)d;
        for (int b = l; b >= 1; b--) {
            const long double dm = (-2.0L * a * d - r[b + 1 + l] * dn) / r[b + l];
            dl[(size_t)(a + l) + w * (size_t)(b - 1 + l)] = (double)dm;
            dn = d;
            d = dm;
        }
        const double sg = ((l + a) & 1) ? -1.0 : 1.0;
        for (int b = 1; b <= l; b++)
            dl[(size_t)(a + l) + w * (size_t)(l - b)] = sg * dl[(size_t)(a + l) + w * (size_t)(l + b)];
    }
    free(r);
    free(E);
}

/* The d(pi/2) plane the transforms use: the reference's Turok-Bucher plane
 * unless the diagnostic method is selected. */
static void orc_dl_plane(double *dl, int l)
{
    if (orc_dl_method == 1) orc_dl_edge_ld(dl, l);
    else orc_dl_beta_operator(dl, ORC_PION2, l);
}

/* ------------------------------------------------------------------ */
/* FFT with FFTW's c2r / r2c semantics (the reference calls FFTW3's    */
/* dfftw_plan_dft_c2r_1d / r2c_1d at s2dw_core_mod.f90:511-526 and     */
/* :869-885).  Mixed-radix recursive Cooley-Tukey, naive DFT per prime */
/* factor, twiddles from an exact table.                              */
/* ------------------------------------------------------------------ */

typedef struct { int n; dcx *tw; } orc_fftplan;

static orc_fftplan orc_fft_make(int n, int sign)
{
    orc_fftplan p;
    p.n = n;
    p.tw = (dcx *)malloc(sizeof(dcx) * n);
    for (int k = 0; k < n; k++) {
        double a = 2.0 * ORC_PI * (double)k / (double)n;
        p.tw[k] = cos(a) + I * (sign * sin(a));
    }
    return p;
}

static void orc_fft_free(orc_fftplan *p) { free(p->tw); }

static void orc_fft_rec(const orc_fftplan *P, const dcx *in, int stride, dcx *out, int n, dcx *scratch)
{
    if (n == 1) { out[0] = in[0]; return; }
    int p = 2;
    while (n % p) { p++; if (p * p > n) { p = n; break; } }
    int m = n / p;
    for (int r = 0; r < p; r++) orc_fft_rec(P, in + (size_t)r * stride, stride * p, out + (size_t)r * m, m, scratch);
    int tstep = P->n / n;
    for (int k = 0; k < m; k++) {
        for (int r = 0; r < p; r++)
            scratch[r] = out[(size_t)r * m + k] * P->tw[((size_t)r * k * tstep) % P->n];
        for (int q = 0; q < p; q++) {
            dcx acc = 0.0;
            for (int r = 0; r < p; r++) acc += scratch[r] * P->tw[((size_t)r * q * m * tstep) % P->n];
            scratch[p + q] = acc;
        }
        for (int q = 0; q < p; q++) out[k + (size_t)q * m] = scratch[p + q];
    }
}

/* out[k] = sum_j in[j] exp(sign*2 pi i j k/n) */
static void orc_fft_exec(const orc_fftplan *P, const dcx *in, dcx *out, dcx *scratch)
{
    orc_fft_rec(P, in, 1, out, P->n, scratch);
}

/* ------------------------------------------------------------------ */
/* Analysis: s2dw_core_mod.f90:572-775 (dynamic) / :342-534 (static)   */
/* ------------------------------------------------------------------ */

/* One scale of the analysis.  Fills coeff(0:2bl-2,0:2bl-1,0:N-1) with
 * stride `astride` between consecutive a (1 for the dynamic layout,
 * J+1 for the static layout) and (2B-1)*astride-style strides given by
 * bstride/gstride.  Optional intermediate outputs for stage debugging:
 * Tmmm(0:bl-1,0:bl-1,0:2N-2), Tmmg(0:bl-1,0:bl-1,0:N-1),
 * Tmbg(0:bl-1,0:2bl-1,0:N-1). */
int orc_analysis_scale(int jj, double *out, size_t astride, size_t bstride, size_t gstride,
                       const dcx *flm, const double *K_gamma, const dcx *Slm, int J, int B, int N,
                       double alpha, dcx *dbg_Tmmm, dcx *dbg_Tmmg, dcx *dbg_Tmbg)
{
    int bl_hi, bl_lo;
    orc_band_limits(jj, B, alpha, &bl_hi, &bl_lo);
    const int bl = bl_hi;
    const size_t nT = (size_t)bl * bl;
    dcx *Tmmm = (dcx *)calloc(nT * (2 * N - 1), sizeof(dcx));
    if (!Tmmm) return ORC_ERR_MEM;
#define TMMM(m, mm, k) Tmmm[(m) + (size_t)bl * (mm) + nT * (k)]
    /* HOT LOOP 1: s2dw_core_mod.f90:625-673.  The reference reduces into
     * Tmmm with an OpenMP reduction over el; here each thread owns a
     * private copy and the copies are summed at the end. */
#pragma omp parallel
    {
        dcx *Tp = (dcx *)calloc(nT * (2 * N - 1), sizeof(dcx));
        double *dl = (double *)malloc(sizeof(double) * (size_t)(2 * bl + 1) * (2 * bl + 1));
#pragma omp for schedule(dynamic, 10)
        for (int el = bl_lo + 1; el <= bl_hi - 1; el++) {
            orc_dl_plane(dl, el);
            const size_t w = (size_t)(2 * el + 1);
#define D(i, k) dl[((i) + el) + w * ((k) + el)]
            int kmax = (N - 1) < el ? (N - 1) : el;
            double mmmsign = (kmax % 2 == 0) ? -1.0 : 1.0;
            double Kg = K_gamma[jj + (size_t)(J + 1) * el];
            for (int mmm = -kmax; mmm <= kmax; mmm++) {
                mmmsign = -mmmsign;
                for (int mm = 0; mm <= el; mm++) {
                    for (int m = 0; m <= el; m++) {
                        dcx sb;
                        if (mmm < 0)
                            sb = ((mmmsign * Kg) * Slm[el + (size_t)B * (-mmm)]) * flm[el + (size_t)B * m];
                        else
                            sb = conj(Kg * Slm[el + (size_t)B * mmm]) * flm[el + (size_t)B * m];
                        dcx e = cexp(I * ((double)(mmm - m) * ORC_PION2));
                        Tp[(m) + (size_t)bl * (mm) + nT * (mmm + N - 1)] += ((e * D(mm, m)) * D(mm, mmm)) * sb;
                    }
                }
            }
#undef D
        }
#pragma omp critical
        for (size_t i = 0; i < nT * (2 * N - 1); i++) Tmmm[i] += Tp[i];
        free(Tp);
        free(dl);
    }
    if (dbg_Tmmm) memcpy(dbg_Tmmm, Tmmm, sizeof(dcx) * nT * (2 * N - 1));

    /* gamma DFT: s2dw_core_mod.f90:679-705 */
    dcx *Tmmg = (dcx *)calloc(nT * N, sizeof(dcx));
#pragma omp parallel for collapse(2) schedule(dynamic, 10)
    for (int gg = 0; gg <= N - 1; gg++) {
        for (int mm = 0; mm <= bl - 1; mm++) {
            double gamma_g = ORC_PI * gg / (double)N;
            for (int m = 0; m <= bl - 1; m++) {
                dcx acc = Tmmg[m + (size_t)bl * mm + nT * gg];
                for (int mmm = -(N - 1); mmm <= N - 1; mmm++) {
                    if ((N + mmm) % 2 != 0)
                        acc = acc + TMMM(m, mm, mmm + N - 1) * cexp(I * (mmm * gamma_g));
                }
                Tmmg[m + (size_t)bl * mm + nT * gg] = acc;
            }
        }
    }
#undef TMMM
    free(Tmmm);
    if (dbg_Tmmg) memcpy(dbg_Tmmg, Tmmg, sizeof(dcx) * nT * N);

    /* beta transform (naive, as in the reference): :708-743 */
    const size_t nB = (size_t)bl * 2 * bl;
    dcx *Tmbg = (dcx *)calloc(nB * N, sizeof(dcx));
#pragma omp parallel for collapse(2) schedule(dynamic, 10)
    for (int gg = 0; gg <= N - 1; gg++) {
        for (int bb = 0; bb <= 2 * bl - 1; bb++) {
            double beta_b = ORC_PI * (2.0 * bb + 1.0) / (4.0 * bl);
            for (int mm = 0; mm <= bl - 1; mm++) {
                double cb = 2.0 * cos(mm * beta_b), sbv = 2.0 * sin(mm * beta_b);
                for (int m = 0; m <= bl - 1; m++) {
                    dcx eta;
                    if (mm == 0) eta = 1.0;
                    else if ((m + N - 1) % 2 == 0) eta = cb;
                    else eta = I * sbv;
                    Tmbg[m + (size_t)bl * bb + nB * gg] += Tmmg[m + (size_t)bl * mm + nT * gg] * eta;
                }
            }
        }
    }
    free(Tmmg);
    if (dbg_Tmbg) memcpy(dbg_Tmbg, Tmbg, sizeof(dcx) * nB * N);

    /* alpha c2r FFT (FFTW semantics: unnormalised, +i, Im X0 ignored),
     * s2dw_core_mod.f90:746-768 */
    const int n = 2 * bl - 1;
    orc_fftplan P = orc_fft_make(n, +1);
#pragma omp parallel
    {
        dcx *x = (dcx *)malloc(sizeof(dcx) * n), *y = (dcx *)malloc(sizeof(dcx) * n);
        dcx *scr = (dcx *)malloc(sizeof(dcx) * 2 * (n + 1));
#pragma omp for collapse(2) schedule(dynamic, 10)
        for (int gg = 0; gg <= N - 1; gg++) {
            for (int bb = 0; bb <= 2 * bl - 1; bb++) {
                const dcx *X = Tmbg + (size_t)bl * bb + nB * gg;
                x[0] = creal(X[0]);
                for (int m = 1; m < bl; m++) { x[m] = X[m]; x[n - m] = conj(X[m]); }
                orc_fft_exec(&P, x, y, scr);
                for (int a = 0; a < n; a++) out[astride * a + bstride * bb + gstride * gg] = creal(y[a]);
            }
        }
        free(x); free(y); free(scr);
    }
    orc_fft_free(&P);
    free(Tmbg);
    return ORC_OK;
}

/* s2dw_core_analysis_flm2wav_dynamic: wav[jj] points at the per-scale
 * array coeff(0:2bl-2,0:2bl-1,0:N-1). */
int orc_analysis_dynamic(double *const *wav, dcx *scoeff, const dcx *flm, const double *K_gamma,
                         const dcx *Slm, int J, int B, int N, int bl_scoeff, double alpha)
{
    for (int jj = 0; jj <= J; jj++)
        if (!wav[jj]) return ORC_ERR_MEM;
    for (int jj = 0; jj <= J; jj++) {
        int hi, lo;
        orc_band_limits(jj, B, alpha, &hi, &lo);
        size_t n = (size_t)(2 * hi - 1);
        int st = orc_analysis_scale(jj, wav[jj], 1, n, n * 2 * hi, flm, K_gamma, Slm, J, B, N, alpha,
                                    NULL, NULL, NULL);
        if (st) return st;
    }
    for (int m = 0; m < bl_scoeff; m++)
        for (int l = 0; l < bl_scoeff; l++) scoeff[l + (size_t)bl_scoeff * m] = flm[l + (size_t)B * m];
    return ORC_OK;
}

/* s2dw_core_analysis_flm2wav (static layout, jj fastest), :342-534.  Only
 * the region a<2bl-1, b<2bl of each scale is written. */
int orc_analysis_static(double *wav, dcx *scoeff, const dcx *flm, const double *K_gamma,
                        const dcx *Slm, int J, int B, int N, int bl_scoeff, double alpha)
{
    const size_t J1 = (size_t)(J + 1);
    for (int jj = 0; jj <= J; jj++) {
        int st = orc_analysis_scale(jj, wav + jj, J1, J1 * (2 * B - 1), J1 * (2 * B - 1) * 2 * B, flm,
                                    K_gamma, Slm, J, B, N, alpha, NULL, NULL, NULL);
        if (st) return st;
    }
    for (int m = 0; m < bl_scoeff; m++)
        for (int l = 0; l < bl_scoeff; l++) scoeff[l + (size_t)bl_scoeff * m] = flm[l + (size_t)B * m];
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* Synthesis: s2dw_core_mod.f90:1060-1266 (dynamic) / :816-1019        */
/* ------------------------------------------------------------------ */

/* One scale of the synthesis, accumulating into flm.  The scale's
 * wavelet coefficients are read with strides astride/bstride/gstride. */
int orc_synthesis_scale(int jj, dcx *flm, const double *in, size_t astride, size_t bstride,
                        size_t gstride, const double *K_gamma, const dcx *Slm, int J, int B, int N,
                        double alpha, dcx *dbg_V, dcx *dbg_Vmmm)
{
    int bl_hi, bl_lo;
    orc_band_limits(jj, B, alpha, &bl_hi, &bl_lo);
    const int bl = bl_hi, n = 2 * bl - 1;
    const size_t nB = (size_t)bl * 2 * bl;
    /* Step 1, alpha r2c FFT, :1104-1130 */
    dcx *V = (dcx *)calloc(nB * N, sizeof(dcx));
    if (!V) return ORC_ERR_MEM;
#define VV(m, k, p) V[(m) + (size_t)bl * (k) + nB * (p)]
    orc_fftplan P = orc_fft_make(n, -1);
    const double c1 = 4.0 * (ORC_PI * ORC_PI) / (double)N, c2 = 2.0 * bl - 1.0;
#pragma omp parallel
    {
        dcx *x = (dcx *)malloc(sizeof(dcx) * n), *y = (dcx *)malloc(sizeof(dcx) * n);
        dcx *scr = (dcx *)malloc(sizeof(dcx) * 2 * (n + 1));
#pragma omp for collapse(2) schedule(dynamic, 10)
        for (int gg = 0; gg <= N - 1; gg++) {
            for (int bb = 0; bb <= 2 * bl - 1; bb++) {
                for (int a = 0; a < n; a++) x[a] = in[astride * a + bstride * bb + gstride * gg];
                orc_fft_exec(&P, x, y, scr);
                for (int m = 0; m < bl; m++) VV(m, bb, gg) = y[m] * c1 / c2;
            }
        }
        free(x); free(y); free(scr);
    }
    orc_fft_free(&P);
    if (dbg_V) memcpy(dbg_V, V, sizeof(dcx) * nB * N);

    /* Step 2a, gamma: Umnb(0:bl-1,0:N-1,0:2bl-1), :1132-1155 */
    const size_t nU = (size_t)bl * N;
    dcx *U = (dcx *)calloc(nU * 2 * bl, sizeof(dcx));
    for (int gg = 0; gg <= N - 1; gg++) {
        for (int mmm = 0; mmm <= N - 1; mmm++) {
            double gamma_g = ORC_PI * gg / (double)N;
            if ((N + mmm) % 2 != 0) {
                dcx e = cexp(-I * (mmm * gamma_g));
#pragma omp parallel for
                for (int bb = 0; bb < 2 * bl; bb++)
                    for (int m = 0; m < bl; m++)
                        U[m + (size_t)bl * mmm + nU * bb] = U[m + (size_t)bl * mmm + nU * bb] + VV(m, bb, gg) * e;
            }
        }
    }
    /* Step 2b, beta with quadrature weights, :1157-1179 */
    /* zero V(0:bl-1,0:2bl-2,0:N-1) */
    for (int p = 0; p < N; p++)
        for (int k = 0; k <= 2 * bl - 2; k++)
            for (int m = 0; m < bl; m++) VV(m, k, p) = 0.0;
    /* Parallel over mm (each output column is owned by one thread); for
     * every output the b sum runs in the reference's order. */
    double *wq = (double *)malloc(sizeof(double) * 2 * bl);
    for (int bb = 0; bb < 2 * bl; bb++) wq[bb] = orc_quad_weights(ORC_PI * (2.0 * bb + 1.0) / (4.0 * bl), bl);
#pragma omp parallel for collapse(2) schedule(dynamic, 10)
    for (int mmm = 0; mmm <= N - 1; mmm++) {
        for (int mm = -(bl - 1); mm <= bl - 1; mm++) {
            if ((N + mmm) % 2 == 0) continue;
            for (int bb = 0; bb <= 2 * bl - 1; bb++) {
                double beta_b = ORC_PI * (2.0 * bb + 1.0) / (4.0 * bl);
                dcx e = cexp(-(I * (mm * beta_b)));
                for (int m = 0; m < bl; m++)
                    VV(m, mm + bl - 1, mmm) = VV(m, mm + bl - 1, mmm) + (U[m + (size_t)bl * mmm + nU * bb] * wq[bb]) * e;
            }
        }
    }
    free(wq);
    free(U);
    /* Step 3a, fold m' and -m', :1181-1198 */
    for (int mmm = 0; mmm <= N - 1; mmm++) {
        if ((N + mmm) % 2 == 0) continue;
        for (int mm = 1; mm <= bl - 1; mm++)
            for (int m = 0; m < bl; m++)
                VV(m, mm + bl - 1, mmm) = VV(m, mm + bl - 1, mmm) + (double)(((m + mmm) % 2) ? -1 : 1) * VV(m, -mm + bl - 1, mmm);
    }
    if (dbg_Vmmm) memcpy(dbg_Vmmm, V, sizeof(dcx) * nB * N);

    /* Step 3b, Wigner coefficients, :1200-1226 */
    dcx *wig = (dcx *)calloc((size_t)bl * bl * N, sizeof(dcx));
#define WIG(el, m, p) wig[(el) + (size_t)bl * (m) + (size_t)bl * bl * (p)]
#pragma omp parallel
    {
        double *dl = (double *)malloc(sizeof(double) * (size_t)(2 * bl + 1) * (2 * bl + 1));
#pragma omp for schedule(dynamic, 10)
        for (int el = bl_lo + 1; el <= bl_hi - 1; el++) {
            orc_dl_plane(dl, el);
            const size_t w = (size_t)(2 * el + 1);
#define D(i, k) dl[((i) + el) + w * ((k) + el)]
            int kmax = (N - 1) < el ? (N - 1) : el;
            for (int mmm = 0; mmm <= kmax; mmm++) {
                for (int m = 0; m <= el; m++) {
                    if ((N + mmm) % 2 != 0) {
                        dcx s = 0.0;
                        for (int mm = 0; mm <= el; mm++) s = s + (VV(m, mm + bl - 1, mmm) * D(mm, m)) * D(mm, mmm);
                        WIG(el, m, mmm) = s * cexp(-(I * ((double)(mmm - m) * ORC_PION2)));
                    }
                }
            }
#undef D
        }
        free(dl);
    }
#undef VV
    free(V);
    /* harmonic accumulation, :1228-1253 */
#pragma omp parallel for schedule(dynamic, 10)
    for (int el = bl_lo + 1; el <= bl_hi - 1; el++) {
        double Kg = K_gamma[jj + (size_t)(J + 1) * el];
        int kmax = (N - 1) < el ? (N - 1) : el;
        for (int mmm = 0; mmm <= kmax; mmm++) {
            for (int m = 0; m <= el; m++) {
                if (mmm == 0) {
                    flm[el + (size_t)B * m] = flm[el + (size_t)B * m] +
                        (((double)(2 * el + 1) / (8.0 * ORC_PI * ORC_PI)) * WIG(el, m, 0)) * Kg * Slm[el];
                } else if ((N + mmm) % 2 != 0) {
                    flm[el + (size_t)B * m] = flm[el + (size_t)B * m] +
                        ((2.0 * ((double)(2 * el + 1) / (8.0 * ORC_PI * ORC_PI))) * WIG(el, m, mmm)) * Kg *
                            Slm[el + (size_t)B * mmm];
                }
            }
        }
    }
#undef WIG
    free(wig);
    return ORC_OK;
}

static void orc_add_scaling(dcx *flm, const dcx *scoeff, const double *Phi2, int B, int bl_scoeff)
{
    /* :1257-1261 */
    for (int el = 0; el < bl_scoeff; el++)
        for (int m = 0; m < bl_scoeff; m++)
            flm[el + (size_t)B * m] = flm[el + (size_t)B * m] + Phi2[el] * scoeff[el + (size_t)bl_scoeff * m];
}

/* s2dw_core_synthesis_wav2flm_dynamic: wav[jj] points at the per-scale
 * coeff array.  (The reference also frees the arrays; the caller owns
 * them here.) */
int orc_synthesis_dynamic(dcx *flm, double *const *wav, const dcx *scoeff, const double *K_gamma,
                          const double *Phi2, const dcx *Slm, int J, int B, int N, int bl_scoeff,
                          double alpha)
{
    for (int jj = 0; jj <= J; jj++)
        if (!wav[jj]) return ORC_ERR_MEM;
    for (size_t i = 0; i < (size_t)B * B; i++) flm[i] = 0.0;
    for (int jj = 0; jj <= J; jj++) {
        int hi, lo;
        orc_band_limits(jj, B, alpha, &hi, &lo);
        size_t n = (size_t)(2 * hi - 1);
        int st = orc_synthesis_scale(jj, flm, wav[jj], 1, n, n * 2 * hi, K_gamma, Slm, J, B, N, alpha,
                                     NULL, NULL);
        if (st) return st;
    }
    orc_add_scaling(flm, scoeff, Phi2, B, bl_scoeff);
    return ORC_OK;
}

/* s2dw_core_synthesis_wav2flm (static layout), :816-1019 */
int orc_synthesis_static(dcx *flm, const double *wav, const dcx *scoeff, const double *K_gamma,
                         const double *Phi2, const dcx *Slm, int J, int B, int N, int bl_scoeff,
                         double alpha)
{
    const size_t J1 = (size_t)(J + 1);
    for (size_t i = 0; i < (size_t)B * B; i++) flm[i] = 0.0;
    for (int jj = 0; jj <= J; jj++) {
        int st = orc_synthesis_scale(jj, flm, wav + jj, J1, J1 * (2 * B - 1), J1 * (2 * B - 1) * 2 * B,
                                     K_gamma, Slm, J, B, N, alpha, NULL, NULL);
        if (st) return st;
    }
    orc_add_scaling(flm, scoeff, Phi2, B, bl_scoeff);
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* s2dw_test's generator: src/prog/s2dw_test.f90:192-285              */
/* ------------------------------------------------------------------ */

static int32_t orc_ran2_idum2 = 123456789, orc_ran2_iy = 0;
static int32_t orc_ran2_iv[32];

void orc_ran2_reset(void)
{
    orc_ran2_idum2 = 123456789;
    orc_ran2_iy = 0;
    memset(orc_ran2_iv, 0, sizeof(orc_ran2_iv));
}

/* ran2_dp, s2dw_test.f90:247-285.  AM, EPS and RNMX are single-precision
 * parameter expressions in the reference. */
double orc_ran2_dp(int32_t *idum)
{
    const int32_t IM1 = 2147483563, IM2 = 2147483399, IMM1 = IM1 - 1, IA1 = 40014, IA2 = 40692,
                  IQ1 = 53668, IQ2 = 52774, IR1 = 12211, IR2 = 3791, NTAB = 32, NDIV = 1 + IMM1 / NTAB;
    const double AM = (double)(1.0f / (float)IM1);
    const double RNMX = (double)(1.0f - 1.2e-7f);
    int32_t j, k;
    if (*idum <= 0) {
        *idum = (-*idum) > 1 ? -*idum : 1;
        orc_ran2_idum2 = *idum;
        for (j = NTAB + 8; j >= 1; j--) {
            k = *idum / IQ1;
            *idum = IA1 * (*idum - k * IQ1) - k * IR1;
            if (*idum < 0) *idum += IM1;
            if (j <= NTAB) orc_ran2_iv[j - 1] = *idum;
        }
        orc_ran2_iy = orc_ran2_iv[0];
    }
    k = *idum / IQ1;
    *idum = IA1 * (*idum - k * IQ1) - k * IR1;
    if (*idum < 0) *idum += IM1;
    k = orc_ran2_idum2 / IQ2;
    orc_ran2_idum2 = IA2 * (orc_ran2_idum2 - k * IQ2) - k * IR2;
    if (orc_ran2_idum2 < 0) orc_ran2_idum2 += IM2;
    j = 1 + orc_ran2_iy / NDIV;
    orc_ran2_iy = orc_ran2_iv[j - 1] - orc_ran2_idum2;
    orc_ran2_iv[j - 1] = *idum;
    if (orc_ran2_iy < 1) orc_ran2_iy += IMM1;
    double r = AM * orc_ran2_iy;
    return r < RNMX ? r : RNMX;
}

/* s2dw_test_gen_flm, s2dw_test.f90:192-224: flm(0:L,0:L) */
void orc_test_gen_flm(int L, dcx *flm, int32_t seed)
{
    int32_t idum = seed;
    size_t n = (size_t)(L + 1);
    for (size_t i = 0; i < n * n; i++) flm[i] = 0.0;
    for (int el = 0; el <= L; el++) {
        flm[el] = 2.0 * orc_ran2_dp(&idum) - 1.0;
        for (int m = 1; m <= el; m++) {
            double re = 2.0 * orc_ran2_dp(&idum) - 1.0;
            double im = 2.0 * orc_ran2_dp(&idum) - 1.0;
            flm[el + n * m] = re + I * im;
        }
    }
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------------
 * s2dw_stat_moments (src/mod/s2dw_stat_mod.f90:81-275), per scale jj:
 * band limits as :108-118; optional mask applied to the coefficients in
 * place (:121-125) and nj = nint(sum(mask)) (:128-132); nj < 2 is an error
 * (:133-136); mean and the sums of powers 1..6 of s = w - mean over the
 * samples with |mask - 1| < TOL_ZERO (all samples without a mask), summed in
 * array order like Fortran's sum (:147-195, :199-242); variance with the n-1
 * correction (:196, :244); zero variance (< TOL_ZERO) sets the higher moments
 * to zero and raises the ARTH_WARNING code (:248-257); otherwise the
 * standardisations of :259-268.  five / six may be NULL (optional).
 * Returns 0, S2DW_ERROR_ARTH_WARNING (6) or S2DW_ERROR_SIZE_INVALID (8).
 * ------------------------------------------------------------------------ */
int orc_stat_moments(double *const *wav, int J, int B, int N, double alpha, double *mean, double *var,
                     double *skew, double *kur, const double *const *mask, double *five, double *six)
{
    const double TOL_ZERO = 1e-12;
    int status = 0;
    for (int jj = 0; jj <= J; jj++) {
        int hi, lo;
        orc_band_limits(jj, B, alpha, &hi, &lo);
        const long long n = (long long)(2 * hi - 1) * (2 * hi) * N;
        double *w = wav[jj];
        const double *mk = mask ? mask[jj] : NULL;
        long long nj;
        if (mk) {
            double sm = 0.0;
            for (long long i = 0; i < n; i++) w[i] *= mk[i];
            for (long long i = 0; i < n; i++) sm += mk[i];
            nj = (long long)llround(sm);
        } else {
            nj = n;
        }
        if (nj < 2) return 8;
        double m = 0.0;
        for (long long i = 0; i < n; i++)
            if (!mk || fabs(mk[i] - 1.0) < TOL_ZERO) m += w[i];
        m /= (double)nj;
        double ep = 0.0, p2 = 0.0, p3 = 0.0, p4 = 0.0, p5 = 0.0, p6 = 0.0;
        for (long long i = 0; i < n; i++) {
            if (mk && !(fabs(mk[i] - 1.0) < TOL_ZERO)) continue;
            const double s = w[i] - m;
            double p = s * s;
            ep += s;
            p2 += p;
            p *= s;
            p3 += p;
            p *= s;
            p4 += p;
            p *= s;
            p5 += p;
            p *= s;
            p6 += p;
        }
        const double v = (p2 - ep * ep / (double)nj) / (double)(nj - 1);
        const double sdev = sqrt(v);
        mean[jj] = m;
        var[jj] = v;
        if (v < TOL_ZERO) {
            status = 6;
            skew[jj] = 0.0;
            kur[jj] = 0.0;
            if (five) {
                five[jj] = 0.0;
                if (six) six[jj] = 0.0;
            }
        } else {
            skew[jj] = p3 / ((double)nj * sdev * sdev * sdev);
            kur[jj] = p4 / ((double)nj * v * v) - 3.0;
            if (five) {
                five[jj] = p5 / ((double)nj * sdev * sdev * sdev * sdev * sdev);
                if (six) six[jj] = p6 / ((double)nj * v * v * v) - 15.0;
            }
        }
    }
    return status;
}
