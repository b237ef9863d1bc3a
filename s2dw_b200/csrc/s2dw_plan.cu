// Plans, the plan cache and the C-ABI transform entry points.
//
// A plan holds everything that depends only on (B, N, alpha, J, device):
// the recurrence tables for d^l(pi/2), the chirp-z tables of every scale and
// the device workspaces.  The caller's kernel tables (K_gamma, Phi2, Slm) are
// uploaded per call (s2dwc_plan_set_tables), which folds them into per-scale
// factors kappa(j,l,n).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <array>
#include <cmath>
#include <complex>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "s2dw_internal.h"

using namespace s2dw;

struct s2dwc_plan {
    int B = 0, Bp = 0, N = 0, J = 0, device = 0, form = 0, NP = 0;
    double alpha = 0.0;
    int nq[S2DW_NPMAX] = {};
    int hn = 8;  // n rows of H
    int bl_scoeff = 0;
    bool tables_set = false;
    std::vector<int> bl, blo;
    std::vector<long long> wav_off;  // J+2 entries
    // recurrence tables
    double *Om = nullptr, *Acoef = nullptr, *Stm = nullptr, *Gam = nullptr, *Bcoef = nullptr,
           *Em = nullptr, *H = nullptr;
    int32_t *Ste = nullptr, *Ee = nullptr;
    // per-scale transform tables: [scale][CztMode], and the beta modes used
    std::vector<std::array<CztDev, 6>> czt;
    std::vector<int> ana_beta_mode, syn_beta_mode;
    std::map<int, TwDev> tw;
    std::vector<double *> wq;  // quadrature weights per scale
    // caller tables folded into per-scale factor tables
    double *kappaA = nullptr, *kappaS = nullptr, *Phi2 = nullptr;
    double *Ga = nullptr, *Gsyn = nullptr;       // all scales, see LwalkArgs/MwalkArgs
    // a general complex Slm, S = eta (a + i b) with b != 0: the tables of b
    // (built on first use); the contractions then run twice (acc_imag)
    bool slm_general = false;
    long long ga_total = 0, gs_total = 0;
    double *kappaA_b = nullptr, *kappaS_b = nullptr, *Ga_b = nullptr, *Gsyn_b = nullptr;
    std::vector<long long> ga_off, gs_off;       // per-scale offsets (doubles)
    std::vector<int> ga_stride, gs_stride;
    // synthesis tables transposed for the two-l-per-thread m'-walk (MwalkArgs::GT),
    // when the plan's tiles are 64 l high: per scale roundup(bl, 8) x (NP+1) rows
    // of gt_ld[j] = roundup(bl-blo-1, 64) values
    int mw_tile_l = 32, mw_tile_m = 16;
    double *GsT = nullptr, *GsT_b = nullptr;
    long long gt_total = 0;
    std::vector<long long> gt_off;
    std::vector<int> gt_ld;
    double2 *Fw = nullptr;                       // per-call F table [l*Bp + m]
    // per-scale workspaces (scales run concurrently on their own streams):
    // A_j holds Tb / V (N x bl x 2bl), C_j holds Tg (N x bl x bl) / V2f,
    // P_j the scale's flm rows (bl-blo-1) x bl
    double2 *wsA = nullptr, *wsC = nullptr, *wsP = nullptr;
    std::vector<long long> offA, offC, offP;
    std::vector<cudaStream_t> streams;
    std::vector<int2 *> lw_tiles, mw_tiles;   // per-scale tile lists (device)
    std::vector<int> lw_ntiles, mw_ntiles;
    cudaEvent_t ev_fork = nullptr;
    std::vector<cudaEvent_t> ev_join;
    // device buffers of the host-buffer entry points (allocated on first use)
    double *hbWav = nullptr;
    double2 *hbFlm = nullptr, *hbSc = nullptr;
    int hbSc_n = 0;
    // two page-locked staging buffers for pageable caller arrays (first use)
    char *stage[2] = {nullptr, nullptr};
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};
    // host-buffer entry points: the caller's tables last folded in (compared
    // by content, so that repeated calls with the same K_gamma and Slm keep
    // the device tables), a copy stream, and per-scale events that order the
    // copies against the scales' kernels (created on first use)
    std::vector<double> hc_K, hc_S, hc_Phi2;
    int hc_bls = -1;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_host = nullptr;
    std::vector<cudaEvent_t> ev_done, ev_copy;
    long long ws_bytes = 0;
    // optional per-kernel CUDA-event timing: (kind, start, stop) per launch
    bool timing = false;
    std::vector<std::tuple<int, cudaEvent_t, cudaEvent_t>> tev;
    double t_ms[S2DWC_KIND_COUNT] = {0};
    long long t_n[S2DWC_KIND_COUNT] = {0};
    // split-precision form (S2DWC_FORM_SPLIT): built on first use
    struct SplitScale {
        int c0 = 0, nch = 0, ntiles = 0;
        int2 *tiles = nullptr;
        long long dexp_off = 0;
        // synthesis
        int snch = 0, sntiles = 0;
        int2 *stiles = nullptr;
        long long sexp_off = 0;
        // per-scale workspaces (offsets in elements of the buffers below;
        // tg_off and v2f_off count per map: the scale's region of a buffer
        // that holds `sp_cap` maps starts at sp_cap * offset)
        long long fdig_off = 0, vdig_off = 0, fexp_off = 0, tg_off = 0, tb_off = 0, v2f_off = 0, vstride = 0;
    };
    std::vector<SplitScale> sp;
    bool sp_alloc = false, sp_dexp_valid = false;
    int16_t *sp_dexp = nullptr;
    int32_t *sp_fexp = nullptr;
    uint8_t *sp_fdig = nullptr;
    double2 *sp_Tg = nullptr, *sp_Tb = nullptr, *sp_ph = nullptr;
    int16_t *sp_sexp = nullptr;
    int32_t *sp_vexp = nullptr;
    uint8_t *sp_vdig = nullptr;
    double2 *sp_V2f = nullptr, *sp_part = nullptr;
    long long sp_pstride = 0;
    // maps the map-proportional workspaces (Tg, V2f, part) hold: grown on
    // demand up to the 32 maps of one tensor-core pass
    int sp_cap = 0;
    long long sp_tg_map = 0, sp_v2f_map = 0;
    int *sp_err = nullptr;
    unsigned long long sp_wait_ns = 2000000000ull;  // bound on every split-kernel pipeline wait (2 s)
    int sp_min_batch = 1;  // split-form batches smaller than this run the FP64 path
    // moments of the coefficients (built on first use): 32 maps per pass
    double *st_part = nullptr, *st_mean = nullptr;
    int *st_flags = nullptr;
    std::vector<void *> allocs;
    std::mutex mu;  // serialises use of the workspaces
    // footprint-only build (s2dwc_plan_footprint, the memory limit check of
    // s2dwc_plan_create): allocations are counted, nothing touches a device
    bool dry = false;

    ~s2dwc_plan()
    {
        if (dry) return;
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(device);
        for (auto &t : tev) {
            cudaEventDestroy(std::get<1>(t));
            cudaEventDestroy(std::get<2>(t));
        }
        for (auto st : streams) cudaStreamDestroy(st);
        for (auto ev : ev_join) cudaEventDestroy(ev);
        if (ev_fork) cudaEventDestroy(ev_fork);
        for (auto ev : ev_done) cudaEventDestroy(ev);
        for (auto ev : ev_copy) cudaEventDestroy(ev);
        if (ev_host) cudaEventDestroy(ev_host);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        for (void *p : allocs) cudaFree(p);
        for (int i = 0; i < 2; i++) {
            if (stage[i]) cudaFreeHost(stage[i]);
            if (stage_ev[i]) cudaEventDestroy(stage_ev[i]);
        }
        cudaSetDevice(cur);
    }
};

namespace {

// Process-wide limit on the device bytes one plan may hold (0: none), set by
// s2dwc_set_plan_memory_limit.
std::atomic<long long> g_plan_mem_limit{0};

template <typename T>
int dev_alloc(s2dwc_plan *p, T **ptr, size_t count)
{
    void *v = nullptr;
    if (count == 0) count = 1;
    if (p->dry) {
        p->ws_bytes += (long long)(count * sizeof(T));
        *ptr = nullptr;
        return S2DWC_OK;
    }
    const long long lim = g_plan_mem_limit.load();
    if (lim > 0 && p->ws_bytes + (long long)(count * sizeof(T)) > lim)
        return set_error(S2DWC_ERROR_MEM_ALLOC_FAIL,
                         "plan memory limit: %zu more bytes would take the plan to %lld bytes, above the "
                         "limit of %lld", count * sizeof(T), p->ws_bytes + (long long)(count * sizeof(T)), lim);
    cudaError_t e = cudaMalloc(&v, count * sizeof(T));
    if (e != cudaSuccess)
        return set_error(S2DWC_ERROR_MEM_ALLOC_FAIL, "cudaMalloc of %zu bytes failed: %s",
                         count * sizeof(T), cudaGetErrorString(e));
    p->allocs.push_back(v);
    p->ws_bytes += (long long)(count * sizeof(T));
    *ptr = static_cast<T *>(v);
    return S2DWC_OK;
}

// Frees a buffer of `count` elements allocated by dev_alloc.
template <typename T>
void dev_release(s2dwc_plan *p, T **ptr, size_t count)
{
    if (!*ptr) return;
    for (size_t i = 0; i < p->allocs.size(); i++)
        if (p->allocs[i] == static_cast<void *>(*ptr)) {
            p->allocs.erase(p->allocs.begin() + (long)i);
            break;
        }
    cudaFree(*ptr);
    p->ws_bytes -= (long long)(std::max<size_t>(count, 1) * sizeof(T));
    *ptr = nullptr;
}

template <typename T>
int dev_upload(s2dwc_plan *p, T **ptr, const std::vector<T> &h)
{
    int st = dev_alloc(p, ptr, h.size());
    if (st) return st;
    if (p->dry) return S2DWC_OK;
    S2DW_CUDA_TRY(cudaMemcpy(*ptr, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return S2DWC_OK;
}

// Twiddle tables of FFT length M, built with the plan: a status instead of an
// exception (std::map::at) or a default entry (operator[]) if one is missing.
int plan_tw(const s2dwc_plan *p, int M, TwDev *out)
{
    auto it = p->tw.find(M);
    if (it == p->tw.end())
        return set_error(S2DWC_ERROR_ARG_INVALID, "no twiddle table of length %d in the plan (B=%d N=%d)", M, p->B,
                         p->N);
    *out = it->second;
    return S2DWC_OK;
}

int plan_build(s2dwc_plan *p)
{
    const int B = p->B, N = p->N, J = p->J;
    p->NP = positive_nset(N, p->nq);
    p->bl.resize(J + 1);
    p->blo.resize(J + 1);
    p->wav_off.assign(J + 2, 0);
    for (int j = 0; j <= J; j++) {
        band_limits(j, B, p->alpha, &p->bl[j], &p->blo[j]);
        p->wav_off[j + 1] = p->wav_off[j] + (long long)(2 * p->bl[j] - 1) * (2 * p->bl[j]) * N;
    }
    // host tables depend only on B and the rows of H (8, or 16 for N > 8):
    // build once per process
    static std::mutex rec_mu;
    static std::map<int, std::shared_ptr<RecTables>> rec_cache;
    std::shared_ptr<RecTables> tp;
    const int hn = N > 8 ? S2DW_NMAX : 8;
    {
        std::lock_guard<std::mutex> g(rec_mu);
        const int key = B * 64 + hn;
        auto it = rec_cache.find(key);
        if (it == rec_cache.end()) {
            tp = std::make_shared<RecTables>();
            build_rec_tables(B, hn, *tp);
            rec_cache[key] = tp;
        } else {
            tp = it->second;
        }
    }
    p->hn = hn;
    const RecTables &t = *tp;
    // row-padded copies (stride Bp) of the tables read by 32-wide tiles
    const int Bp = (B + 31) / 32 * 32;
    p->Bp = Bp;
    auto pad = [&](const std::vector<double> &v) {
        std::vector<double> o((size_t)B * Bp, 0.0);
        for (int l = 0; l < B; l++)
            std::copy(v.begin() + (size_t)l * B, v.begin() + (size_t)(l + 1) * B, o.begin() + (size_t)l * Bp);
        return o;
    };
    int st;
    if ((st = dev_upload(p, &p->Om, pad(t.Om))) || (st = dev_upload(p, &p->Acoef, pad(t.Acoef))) ||
        (st = dev_upload(p, &p->Stm, t.Stm)) || (st = dev_upload(p, &p->Ste, t.Ste)) ||
        (st = dev_upload(p, &p->Gam, pad(t.Gam))) || (st = dev_upload(p, &p->Bcoef, pad(t.Bcoef))) ||
        (st = dev_upload(p, &p->Em, t.Em)) || (st = dev_upload(p, &p->Ee, t.Ee)) ||
        (st = dev_upload(p, &p->H, t.H)))
        return st;

    // chirp-z tables per scale and mode
    p->czt.resize(J + 1);
    p->wq.resize(J + 1);
    std::map<int, std::array<CztDev, 6>> by_bl;
    std::map<int, double *> wq_by_bl;
    for (int j = 0; j <= J; j++) {
        const int b = p->bl[j], n = 2 * b - 1;
        auto it = by_bl.find(b);
        if (it == by_bl.end()) {
            std::array<CztDev, 6> arr;
            CztSpec specs[4] = {
                {2 * b - 1, 2 * b, 4 * b, +1, -2 * (b - 1), 1, 0},  // CZT_ANA_BETA
                {n, n, n, +1, 0, 0, 0},                              // CZT_ANA_ALPHA
                {n, n, n, -1, 0, 0, 0},                              // CZT_SYN_ALPHA
                {2 * b, 2 * b - 1, 4 * b, -1, 1, -2 * (b - 1), 0},  // CZT_SYN_BETA
            };
            for (int md = 0; md < 4; md++) {
                CztSpec c = specs[md];
                c.M = czt_size(c.K, c.Bout);
                std::vector<double2> pre, post, Hf;
                build_czt_tables(c, pre, post, Hf);
                CztDev d;
                d.M = c.M;
                d.spec = c;
                if ((st = dev_upload(p, &d.pre, pre)) || (st = dev_upload(p, &d.Hf, Hf))) return st;
                // the alpha stages' two chirps are the same table (K = Bout,
                // no offsets): one copy, so that the kernels' table reads
                // share their L1 lines
                if (c.K == c.Bout && c.k0x2 == c.b0x2) {
                    d.post = d.pre;
                } else if ((st = dev_upload(p, &d.post, post))) {
                    return st;
                }
                arr[md] = d;
                if (!p->tw.count(c.M)) {
                    std::vector<double2> hi, lo;
                    build_twiddles(c.M, hi, lo);
                    TwDev tw;
                    tw.M = c.M;
                    if ((st = dev_upload(p, &tw.hi, hi)) || (st = dev_upload(p, &tw.lo, lo))) return st;
                    p->tw[c.M] = tw;
                }
            }
            // beta transforms as one power-of-two FFT of length L = 2 bl (a
            // DCT-III / DCT-II pair of that length) when 2 bl is a power of two
            const int L2 = 2 * b;
            if (L2 >= 16 && L2 <= 4096 && (L2 & (L2 - 1)) == 0) {
                std::vector<double2> twb;
                build_beta_twiddles(b, twb);
                for (int md : {(int)FFT_ANA_BETA, (int)FFT_SYN_BETA}) {
                    CztDev d;
                    d.M = L2;
                    d.spec = CztSpec{2 * b, md == FFT_ANA_BETA ? 2 * b : 2 * b - 1, L2, md == FFT_ANA_BETA ? 1 : -1, 0,
                                     0, L2};
                    if ((st = dev_upload(p, &d.pre, twb))) return st;
                    arr[md] = d;
                }
                if (!p->tw.count(L2)) {
                    std::vector<double2> hi, lo;
                    build_twiddles(L2, hi, lo);
                    TwDev tw;
                    tw.M = L2;
                    if ((st = dev_upload(p, &tw.hi, hi)) || (st = dev_upload(p, &tw.lo, lo))) return st;
                    p->tw[L2] = tw;
                }
            }
            it = by_bl.emplace(b, arr).first;
            std::vector<double> w(2 * b);
            for (int bb = 0; bb < 2 * b; bb++)
                w[bb] = quad_weight(M_PI * (2.0 * bb + 1.0) / (4.0 * b), b);
            double *dw;
            if ((st = dev_upload(p, &dw, w))) return st;
            wq_by_bl[b] = dw;
        }
        p->czt[j] = it->second;
        p->wq[j] = wq_by_bl[b];
        const bool fftb = it->second[FFT_ANA_BETA].M > 0;
        p->ana_beta_mode.push_back(fftb ? FFT_ANA_BETA : CZT_ANA_BETA);
        p->syn_beta_mode.push_back(fftb ? FFT_SYN_BETA : CZT_SYN_BETA);
    }
    // kernel-table factors
    if ((st = dev_alloc(p, &p->kappaA, (size_t)(J + 1) * B * p->NP)) ||
        (st = dev_alloc(p, &p->kappaS, (size_t)(J + 1) * B * p->NP)) ||
        (st = dev_alloc(p, &p->Phi2, (size_t)B)))
        return st;
    // per-scale factor tables: rows l in (blo, bl)
    long long na = 0, ns = 0;
    for (int j = 0; j <= J; j++) {
        const int nl = std::max(0, p->bl[j] - p->blo[j] - 1);
        p->ga_stride.push_back((p->bl[j] + 31) / 32 * 32);
        p->gs_stride.push_back((p->bl[j] + 7) / 8 * 8);
        p->ga_off.push_back(na);
        p->gs_off.push_back(ns);
        na += (long long)nl * p->NP * p->ga_stride[j];
        ns += (long long)nl * p->NP * p->gs_stride[j];
    }
    p->ga_total = na;
    p->gs_total = ns;
    p->mw_tile_l = mwalk_tile_l(p->NP);
    p->mw_tile_m = mwalk_tile_m(p->NP);
    if (p->mw_tile_l == 64) {
        long long nt = 0;
        for (int j = 0; j <= J; j++) {
            const int nl = std::max(0, p->bl[j] - p->blo[j] - 1);
            p->gt_ld.push_back((nl + 63) / 64 * 64);
            p->gt_off.push_back(nt);
            nt += (long long)(p->bl[j] + 7) / 8 * 8 * (p->NP + 1) * p->gt_ld[j];
        }
        p->gt_total = nt;
        if ((st = dev_alloc(p, &p->GsT, (size_t)std::max(1LL, nt)))) return st;
    }
    if ((st = dev_alloc(p, &p->Ga, (size_t)std::max(1LL, na))) ||
        (st = dev_alloc(p, &p->Gsyn, (size_t)std::max(1LL, ns))) ||
        (st = dev_alloc(p, &p->Fw, (size_t)B * Bp)))
        return st;
    // per-scale workspaces
    long long nA = 0, nC = 0, nP = 0;
    for (int j = 0; j <= J; j++) {
        const long long b = p->bl[j];
        p->offA.push_back(nA);
        p->offC.push_back(nC);
        p->offP.push_back(nP);
        nA += (long long)N * b * 2 * b;
        nC += std::max((long long)N * b * b, (long long)p->NP * b * p->gs_stride[j]);
        nP += (long long)std::max(0, p->bl[j] - p->blo[j] - 1) * b;
    }
    if ((st = dev_alloc(p, &p->wsA, (size_t)nA)) || (st = dev_alloc(p, &p->wsC, (size_t)nC)) ||
        (st = dev_alloc(p, &p->wsP, (size_t)std::max(1LL, nP))))
        return st;
    for (int j = 0; j <= J; j++) {
        std::vector<int2> tl;
        build_lwalk_tiles(p->bl[j], p->blo[j], lwalk_tile_m(p->NP), tl);
        int2 *d = nullptr;
        if ((st = dev_upload(p, &d, tl))) return st;
        p->lw_tiles.push_back(d);
        p->lw_ntiles.push_back((int)tl.size());
        build_mwalk_tiles(p->bl[j], p->blo[j], p->mw_tile_m, p->mw_tile_l, tl);
        d = nullptr;
        if (tl.empty()) tl.push_back(make_int2(0, 0));  // keep a valid allocation
        if ((st = dev_upload(p, &d, tl))) return st;
        p->mw_tiles.push_back(d);
        p->mw_ntiles.push_back(p->bl[j] - p->blo[j] - 1 > 0 ? (int)tl.size() : 0);
    }
    if (p->dry) return S2DWC_OK;
    if ((std::find(p->bl.begin(), p->bl.end(), 1024) != p->bl.end() ||
         std::find(p->bl.begin(), p->bl.end(), 256) != p->bl.end()) &&
        (st = pfa_prepare()))
        return st;
    p->streams.resize(J + 1);
    p->ev_join.resize(J + 1);
    for (int j = 0; j <= J; j++) {
        S2DW_CUDA_TRY(cudaStreamCreateWithFlags(&p->streams[j], cudaStreamNonBlocking));
        S2DW_CUDA_TRY(cudaEventCreateWithFlags(&p->ev_join[j], cudaEventDisableTiming));
    }
    S2DW_CUDA_TRY(cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming));
    return S2DWC_OK;
}

std::mutex g_cache_mu;
std::map<std::tuple<int, int, int, int, long long, int>, std::unique_ptr<s2dwc_plan>> g_cache;

int validate_sizes(int B, int N, double alpha, int J)
{
    if (B < 2) return set_error(S2DWC_ERROR_SIZE_INVALID, "B=%d must be >= 2", B);
    if (N < 1 || N > S2DW_NMAX)
        return set_error(S2DWC_ERROR_SIZE_INVALID, "N=%d unsupported (1 <= N <= %d)", N, S2DW_NMAX);
    if (N > B) return set_error(S2DWC_ERROR_SIZE_INVALID, "N=%d exceeds B=%d", N, B);
    if (!(alpha > 1.0)) return set_error(S2DWC_ERROR_SIZE_INVALID, "alpha=%g must exceed 1", alpha);
    if (B > 2048) return set_error(S2DWC_ERROR_SIZE_INVALID, "B=%d exceeds the supported 2048", B);
    if (J > S2DW_JMAX) return set_error(S2DWC_ERROR_SIZE_INVALID, "J=%d exceeds the supported %d", J, S2DW_JMAX);
    if (!params_valid(J, B, alpha, N))
        return set_error(S2DWC_ERROR_SIZE_INVALID, "J=%d invalid for B=%d alpha=%g (1<=J<=%d)", J, B,
                         alpha, comp_jmax(B, alpha));
    return S2DWC_OK;
}

int get_cached_plan(int B, int N, double alpha, int J, s2dwc_plan **out)
{
    int dev = 0;
    S2DW_CUDA_TRY(cudaGetDevice(&dev));
    long long abits;
    std::memcpy(&abits, &alpha, sizeof(abits));
    auto key = std::make_tuple(B, N, J, dev, abits, 0);
    std::lock_guard<std::mutex> g(g_cache_mu);
    auto it = g_cache.find(key);
    if (it != g_cache.end()) {
        *out = it->second.get();
        return S2DWC_OK;
    }
    s2dwc_plan *p = nullptr;
    int st = s2dwc_plan_create(&p, B, N, alpha, J, S2DWC_FORM_FP64, dev);
    if (st) return st;
    g_cache.emplace(key, std::unique_ptr<s2dwc_plan>(p));
    *out = p;
    return S2DWC_OK;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// Brackets one launch with CUDA events on its stream when timing is on.
struct KernelTimer {
    s2dwc_plan *p;
    int kind;
    cudaStream_t s;
    cudaEvent_t a = nullptr, b = nullptr;
    KernelTimer(s2dwc_plan *p_, int k, cudaStream_t s_) : p(p_), kind(k), s(s_)
    {
        if (p->timing && cudaEventCreate(&a) == cudaSuccess && cudaEventCreate(&b) == cudaSuccess)
            cudaEventRecord(a, s);
    }
    ~KernelTimer()
    {
        if (a && b) {
            cudaEventRecord(b, s);
            p->tev.emplace_back(kind, a, b);
        }
    }
};

// Runs the analysis: the F table on `s`, then every scale on its own stream
// (forked from and joined back to `s`).
// Per-scale hook: enqueued on scale j's stream after (analysis) or before
// (synthesis) that scale's kernels; the host-buffer entry points use it to
// overlap each scale's host<->device copy with the other scales' kernels.
using ScaleHook = std::function<int(int, cudaStream_t)>;

// full_band_serial (host-buffer entry points): the scales of the largest band
// limit, which hold most of the coefficients, run one after another, the
// last scale first, so that the first one's device-to-host copy overlaps the
// next one's kernels instead of all of them finishing together at the end.
// (Queuing the smaller scales ahead of them measured 2 % slower end to end.)
int run_analysis(s2dwc_plan *p, double *d_wav, double2 *d_scoeff, const double2 *d_flm, cudaStream_t s,
                 const ScaleHook &after = ScaleHook(), bool full_band_serial = false)
{
    int st;
    {
        KernelTimer kt(p, S2DWC_KIND_OTHER, s);
        if ((st = launch_fprep(p->Fw, d_flm, p->Om, p->B, p->Bp, s))) return st;
    }
    S2DW_CUDA_TRY(cudaEventRecord(p->ev_fork, s));
    const bool serial = full_band_serial && !p->timing && (int)p->ev_done.size() == p->J + 1;
    int prev_full = -1;
    for (int jj = 0; jj <= p->J; jj++) {
        const int j = serial ? p->J - jj : jj;
        // per-kernel timing runs every launch on the caller's stream so that
        // each event pair brackets one kernel running alone
        cudaStream_t sj = p->timing ? s : p->streams[j];
        if (!p->timing) S2DW_CUDA_TRY(cudaStreamWaitEvent(sj, p->ev_fork, 0));
        const int bl = p->bl[j];
        const bool full = serial && bl == p->bl[p->J];
        if (full && prev_full >= 0) S2DW_CUDA_TRY(cudaStreamWaitEvent(sj, p->ev_done[prev_full], 0));
        double2 *Tg = p->wsC + p->offC[j], *Tb = p->wsA + p->offA[j];
        LwalkArgs la{};
        la.B = p->B;
        la.Bp = p->Bp;
        la.N = p->N;
        la.NP = p->NP;
        la.bl = bl;
        la.blo = p->blo[j];
        std::memcpy(la.nq, p->nq, sizeof(la.nq));
        la.Acoef = p->Acoef;
        la.Stm = p->Stm;
        la.Ste = p->Ste;
        la.G = p->Ga + p->ga_off[j];
        la.Gs = p->ga_stride[j];
        la.F = p->Fw;
        la.Tg = Tg;
        la.tiles = p->lw_tiles[j];
        la.ntiles = p->lw_ntiles[j];
        {
            KernelTimer kt(p, S2DWC_KIND_LWALK, sj);
            if ((st = launch_lwalk(la, sj))) return st;
        }
        if (p->slm_general) {  // the b part of a general Slm, accumulated into Tg
            la.G = p->Ga_b + p->ga_off[j];
            la.acc_imag = 1;
            KernelTimer kt(p, S2DWC_KIND_LWALK, sj);
            if ((st = launch_lwalk(la, sj))) return st;
        }
        CztArgs ca{};
        ca.mode = p->ana_beta_mode[j];
        ca.bl = bl;
        ca.N = p->N;
        ca.NP = p->NP;
        std::memcpy(ca.nq, p->nq, sizeof(ca.nq));
        ca.rows = p->N * bl;
        ca.czt = p->czt[j][ca.mode];
        if ((st = plan_tw(p, ca.czt.M, &ca.tw))) return st;
        ca.in_c = Tg;
        ca.out_c = Tb;
        {
            KernelTimer kt(p, S2DWC_KIND_ANA_BETA, sj);
            if ((st = launch_czt(ca, sj))) return st;
        }
        ca.mode = CZT_ANA_ALPHA;
        ca.rows = p->N * bl;  // (g, b pair)
        ca.czt = p->czt[j][CZT_ANA_ALPHA];
        if ((st = plan_tw(p, ca.czt.M, &ca.tw))) return st;
        ca.in_c = Tb;
        ca.out_c = nullptr;
        ca.out_r = d_wav + p->wav_off[j];
        {
            KernelTimer kt(p, S2DWC_KIND_ANA_ALPHA, sj);
            if ((st = launch_czt(ca, sj))) return st;
        }
        if (full) {
            S2DW_CUDA_TRY(cudaEventRecord(p->ev_done[j], sj));
            prev_full = j;
        }
        if (after && (st = after(j, sj))) return st;
        if (!p->timing) S2DW_CUDA_TRY(cudaEventRecord(p->ev_join[j], sj));
    }
    {
        KernelTimer kt(p, S2DWC_KIND_OTHER, s);
        if ((st = launch_scoeff_copy(d_scoeff, d_flm, p->B, p->bl_scoeff, s))) return st;
    }
    if (p->timing) return S2DWC_OK;
    for (int j = 0; j <= p->J; j++) S2DW_CUDA_TRY(cudaStreamWaitEvent(s, p->ev_join[j], 0));
    return S2DWC_OK;
}

// largest_first: scales queued from the last (largest) down, the order in
// which the host-buffer entry points bring the coefficients in.
int run_synthesis(s2dwc_plan *p, double2 *d_flm, const double *d_wav, const double2 *d_scoeff,
                  cudaStream_t s, const ScaleHook &before = ScaleHook(), bool largest_first = false)
{
    int st;
    S2DW_CUDA_TRY(cudaEventRecord(p->ev_fork, s));
    for (int jj = 0; jj <= p->J; jj++) {
        const int j = largest_first ? p->J - jj : jj;
        cudaStream_t sj = p->timing ? s : p->streams[j];
        if (!p->timing) S2DW_CUDA_TRY(cudaStreamWaitEvent(sj, p->ev_fork, 0));
        if (before && (st = before(j, sj))) return st;
        const int bl = p->bl[j];
        double2 *Vw = p->wsA + p->offA[j], *V2f = p->wsC + p->offC[j];
        CztArgs ca{};
        ca.mode = CZT_SYN_ALPHA;
        ca.bl = bl;
        ca.N = p->N;
        ca.NP = p->NP;
        std::memcpy(ca.nq, p->nq, sizeof(ca.nq));
        ca.rows = p->N * bl;
        ca.czt = p->czt[j][CZT_SYN_ALPHA];
        if ((st = plan_tw(p, ca.czt.M, &ca.tw))) return st;
        ca.in_r = d_wav + p->wav_off[j];
        ca.out_c = Vw;
        ca.scale = (4.0 * (M_PI * M_PI) / (double)p->N) / (2.0 * bl - 1.0);
        {
            KernelTimer kt(p, S2DWC_KIND_SYN_ALPHA, sj);
            if ((st = launch_czt(ca, sj))) return st;
        }
        ca.mode = p->syn_beta_mode[j];
        ca.rows = p->NP * bl;
        ca.czt = p->czt[j][ca.mode];
        if ((st = plan_tw(p, ca.czt.M, &ca.tw))) return st;
        ca.in_c = Vw;
        ca.in_r = nullptr;
        ca.out_c = V2f;
        ca.out_stride = p->gs_stride[j];
        ca.wq = p->wq[j];
        {
            KernelTimer kt(p, S2DWC_KIND_SYN_BETA, sj);
            if ((st = launch_czt(ca, sj))) return st;
        }
        MwalkArgs ma{};
        ma.B = p->B;
        ma.Bp = p->Bp;
        ma.N = p->N;
        ma.NP = p->NP;
        ma.bl = bl;
        ma.blo = p->blo[j];
        std::memcpy(ma.nq, p->nq, sizeof(ma.nq));
        ma.Bcoef = p->Bcoef;
        ma.Em = p->Em;
        ma.Ee = p->Ee;
        ma.G = p->Gsyn + p->gs_off[j];
        ma.Gs = p->gs_stride[j];
        ma.V2f = V2f;
        ma.Vs = p->gs_stride[j];
        ma.part = p->wsP + p->offP[j];
        ma.GT = p->GsT ? p->GsT + p->gt_off[j] : nullptr;
        ma.Ts = p->GsT ? p->gt_ld[j] : 0;
        ma.tile_l = p->mw_tile_l;
        ma.tile_m = p->mw_tile_m;
        ma.tiles = p->mw_tiles[j];
        ma.ntiles = p->mw_ntiles[j];
        {
            KernelTimer kt(p, S2DWC_KIND_MWALK, sj);
            if ((st = launch_mwalk(ma, sj))) return st;
        }
        if (p->slm_general) {  // the b part of a general Slm, accumulated into part
            ma.G = p->Gsyn_b + p->gs_off[j];
            if (p->GsT) ma.GT = p->GsT_b + p->gt_off[j];
            ma.acc_imag = 1;
            KernelTimer kt(p, S2DWC_KIND_MWALK, sj);
            if ((st = launch_mwalk(ma, sj))) return st;
        }
        if (!p->timing) S2DW_CUDA_TRY(cudaEventRecord(p->ev_join[j], sj));
    }
    if (!p->timing)
        for (int j = 0; j <= p->J; j++) S2DW_CUDA_TRY(cudaStreamWaitEvent(s, p->ev_join[j], 0));
    CombineArgs cb{};
    cb.B = p->B;
    cb.J = p->J;
    cb.bs = p->bl_scoeff;
    for (int j = 0; j <= p->J; j++) {
        cb.bl[j] = p->bl[j];
        cb.blo[j] = p->blo[j];
        cb.off[j] = p->offP[j];
    }
    cb.parts = p->wsP;
    cb.scoeff = d_scoeff;
    cb.Phi2 = p->Phi2;
    cb.flm = d_flm;
    KernelTimer kt(p, S2DWC_KIND_OTHER, s);
    return launch_combine(cb, s);
}

// Layout of the caller-independent workspace of run_analysis_serial: the F
// table, then one scale's Tg and Tb at the largest band limit, each region
// starting on a 256-byte boundary.
struct SerialLayout {
    long long offTg, offTb, bytes;
};

SerialLayout serial_layout(const s2dwc_plan *p)
{
    auto up = [](long long x) { return (x + 255) / 256 * 256; };
    const long long b = *std::max_element(p->bl.begin(), p->bl.end());
    SerialLayout L;
    L.offTg = up((long long)p->B * p->Bp * (long long)sizeof(double2));
    L.offTb = L.offTg + up((long long)p->N * b * b * (long long)sizeof(double2));
    L.bytes = L.offTb + (long long)p->N * b * 2 * b * (long long)sizeof(double2);
    return L;
}

// The analysis of run_analysis with its F table and per-scale workspaces in
// `ws` (serial_layout bytes) instead of the plan's: every launch on `s`, the
// scales one after another, so that each scale reuses the same Tg and Tb.
// Every element a kernel reads here is written earlier in the same call, so
// `ws` needs no initial contents.
int run_analysis_serial(const s2dwc_plan *p, unsigned char *ws, double *d_wav, double2 *d_scoeff,
                        const double2 *d_flm, cudaStream_t s)
{
    const SerialLayout L = serial_layout(p);
    double2 *F = reinterpret_cast<double2 *>(ws);
    double2 *Tg = reinterpret_cast<double2 *>(ws + L.offTg), *Tb = reinterpret_cast<double2 *>(ws + L.offTb);
    int st;
    if ((st = launch_fprep(F, d_flm, p->Om, p->B, p->Bp, s))) return st;
    for (int j = 0; j <= p->J; j++) {
        const int bl = p->bl[j];
        LwalkArgs la{};
        la.B = p->B;
        la.Bp = p->Bp;
        la.N = p->N;
        la.NP = p->NP;
        la.bl = bl;
        la.blo = p->blo[j];
        std::memcpy(la.nq, p->nq, sizeof(la.nq));
        la.Acoef = p->Acoef;
        la.Stm = p->Stm;
        la.Ste = p->Ste;
        la.G = p->Ga + p->ga_off[j];
        la.Gs = p->ga_stride[j];
        la.F = F;
        la.Tg = Tg;
        la.tiles = p->lw_tiles[j];
        la.ntiles = p->lw_ntiles[j];
        if ((st = launch_lwalk(la, s))) return st;
        if (p->slm_general) {  // the b part of a general Slm, accumulated into Tg
            la.G = p->Ga_b + p->ga_off[j];
            la.acc_imag = 1;
            if ((st = launch_lwalk(la, s))) return st;
        }
        CztArgs ca{};
        ca.mode = p->ana_beta_mode[j];
        ca.bl = bl;
        ca.N = p->N;
        ca.NP = p->NP;
        std::memcpy(ca.nq, p->nq, sizeof(ca.nq));
        ca.rows = p->N * bl;
        ca.czt = p->czt[j][ca.mode];
        if ((st = plan_tw(p, ca.czt.M, &ca.tw))) return st;
        ca.in_c = Tg;
        ca.out_c = Tb;
        if ((st = launch_czt(ca, s))) return st;
        ca.mode = CZT_ANA_ALPHA;
        ca.rows = p->N * bl;
        ca.czt = p->czt[j][CZT_ANA_ALPHA];
        if ((st = plan_tw(p, ca.czt.M, &ca.tw))) return st;
        ca.in_c = Tb;
        ca.out_c = nullptr;
        ca.out_r = d_wav + p->wav_off[j];
        if ((st = launch_czt(ca, s))) return st;
    }
    return launch_scoeff_copy(d_scoeff, d_flm, p->B, p->bl_scoeff, s);
}

// Split form: per-scale workspaces (the scales of a batch run concurrently
// on the plan's streams), tile lists and the per-row exponent tables (the
// latter depend on the kernel tables and are rebuilt after set_tables).
int split_prepare(s2dwc_plan *p, int nmaps, cudaStream_t s)
{
    int st;
    if (p->slm_general)
        return set_error(S2DWC_ERROR_ARG_INVALID,
                         "the split form needs Slm of the form s2dw_core_init_directionality produces (S/eta real)");
    const int NP = p->NP, CH = split_chains(NP), MAPS = split_maps_per_pass(), MC = split_syn_mc(NP);
    if (!p->sp_alloc) {
        p->sp.resize(p->J + 1);
        long long nd = 0, ns = 0, fdig = 0, fexp = 0, tg = 0, tb = 0, v2f = 0, vdig = 0;
        for (int j = 0; j <= p->J; j++) {
            auto &S = p->sp[j];
            const int bl = p->bl[j], blo = p->blo[j], nl = bl - blo - 1;
            const long long Vs = p->gs_stride[j];
            S.c0 = (blo + 1) / 32;
            S.nch = (bl - 1) / 32 - S.c0 + 1;
            S.snch = (bl + MC - 1) / MC;
            S.dexp_off = nd;
            nd += (long long)bl * bl * NP;
            S.sexp_off = ns;
            ns += (long long)bl * bl;
            S.fdig_off = fdig;
            fdig += (split_fdig_bytes(bl, S.nch) + 255) / 256 * 256;
            S.vdig_off = vdig;
            vdig += (split_vdig_bytes(bl, S.snch) + 255) / 256 * 256;
            S.fexp_off = fexp;
            fexp += (long long)bl * 64;
            S.tg_off = tg;
            tg += (long long)p->N * bl * bl;
            S.tb_off = tb;
            tb += (long long)p->N * bl * 2 * bl;
            S.vstride = (long long)NP * bl * Vs;
            S.v2f_off = v2f;
            v2f += S.vstride;
            // analysis tiles (m, chain tile), longest walks (smallest first row) first
            std::vector<int2> tl;
            const int np = (bl + CH - 1) / CH;
            for (int m = 0; m < bl; m++)
                for (int pt = 0; pt < np; pt++) tl.push_back(make_int2(m, pt));
            std::stable_sort(tl.begin(), tl.end(), [CH](int2 a, int2 b) {
                return std::max(a.x, a.y * CH) < std::max(b.x, b.y * CH);
            });
            S.ntiles = (int)tl.size();
            if ((st = dev_upload(p, &S.tiles, tl))) return st;
            // synthesis tiles (m, 128-row l tile), m-major so that the tiles of
            // one m share its map digits in L2
            tl.clear();
            for (int m = 0; m < bl; m++)
                for (int lt = 0; lt * 128 < nl; lt++) {
                    const int lbase = blo + 1 + lt * 128;
                    if (m <= std::min(lbase + 127, bl - 1)) tl.push_back(make_int2(m, lt));
                }
            S.sntiles = (int)tl.size();
            if (tl.empty()) tl.push_back(make_int2(0, 0));
            if ((st = dev_upload(p, &S.stiles, tl))) return st;
        }
        p->sp_pstride = std::max(1LL, p->offP.back() + (long long)std::max(0, p->bl[p->J] - p->blo[p->J] - 1) * p->bl[p->J]);
        if ((st = dev_alloc(p, &p->sp_dexp, (size_t)nd)) || (st = dev_alloc(p, &p->sp_sexp, (size_t)ns)) ||
            (st = dev_alloc(p, &p->sp_fexp, (size_t)fexp)) || (st = dev_alloc(p, &p->sp_vexp, (size_t)fexp)) ||
            (st = dev_alloc(p, &p->sp_fdig, (size_t)fdig)) || (st = dev_alloc(p, &p->sp_vdig, (size_t)vdig)) ||
            (st = dev_alloc(p, &p->sp_Tb, (size_t)tb)) || (st = dev_alloc(p, &p->sp_err, 1)))
            return st;
        p->sp_tg_map = tg;
        p->sp_v2f_map = v2f;
        S2DW_CUDA_TRY(cudaMemsetAsync(p->sp_err, 0, sizeof(int), s));
        // gamma-DFT phases exp(i pi n g / N), [g*16 + n+N-1]
        std::vector<double2> ph((size_t)p->N * 16, make_double2(0.0, 0.0));
        for (int g = 0; g < p->N; g++)
            for (int n = -(p->N - 1); n <= p->N - 1; n++) {
                const long double x = 3.141592653589793238462643383279502884L * (long double)(n * g) / (long double)p->N;
                ph[(size_t)g * 16 + n + p->N - 1] = make_double2((double)cosl(x), (double)sinl(x));
            }
        if ((st = dev_upload(p, &p->sp_ph, ph))) return st;
        p->sp_alloc = true;
    }
    const int need = std::max(1, std::min(MAPS, nmaps));
    if (need > p->sp_cap) {
        // the buffers may still be read by earlier work of this plan
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        S2DW_CUDA_TRY(cudaStreamIsCapturing(s, &cs));
        if (cs != cudaStreamCaptureStatusNone)
            return set_error(S2DWC_ERROR_ARG_INVALID,
                             "split workspaces for %d maps must be sized before graph capture (run the batch once)",
                             need);
        if (p->sp_cap > 0) {
            S2DW_CUDA_TRY(cudaStreamSynchronize(s));
            for (auto st2 : p->streams) S2DW_CUDA_TRY(cudaStreamSynchronize(st2));
        }
        dev_release(p, &p->sp_Tg, (size_t)(p->sp_cap * p->sp_tg_map));
        dev_release(p, &p->sp_V2f, (size_t)(p->sp_cap * p->sp_v2f_map));
        dev_release(p, &p->sp_part, (size_t)(p->sp_cap * p->sp_pstride));
        p->sp_cap = 0;
        if ((st = dev_alloc(p, &p->sp_Tg, (size_t)(need * p->sp_tg_map))) ||
            (st = dev_alloc(p, &p->sp_V2f, (size_t)(need * p->sp_v2f_map))) ||
            (st = dev_alloc(p, &p->sp_part, (size_t)(need * p->sp_pstride))))
            return st;
        p->sp_cap = need;
    }
    if (!p->sp_dexp_valid) {
        for (int j = 0; j <= p->J; j++) {
            SplitArgs a{};
            a.B = p->B;
            a.Bp = p->Bp;
            a.N = p->N;
            a.NP = NP;
            a.bl = p->bl[j];
            a.blo = p->blo[j];
            std::memcpy(a.nq, p->nq, sizeof(a.nq));
            a.Acoef = p->Acoef;
            a.Om = p->Om;
            a.Stm = p->Stm;
            a.Ste = p->Ste;
            a.G = p->Ga + p->ga_off[j];
            a.Gs = p->ga_stride[j];
            a.dexp = p->sp_dexp + p->sp[j].dexp_off;
            a.tiles = p->sp[j].tiles;
            a.ntiles = p->sp[j].ntiles;
            if ((st = launch_split_dexp(a, s))) return st;
            SplitSynArgs b{};
            b.B = p->B;
            b.Bp = p->Bp;
            b.N = p->N;
            b.NP = NP;
            b.bl = p->bl[j];
            b.blo = p->blo[j];
            b.Bcoef = p->Bcoef;
            b.Em = p->Em;
            b.Ee = p->Ee;
            b.G = p->Gsyn + p->gs_off[j];
            b.Gs = p->gs_stride[j];
            b.sexp = p->sp_sexp + p->sp[j].sexp_off;
            b.tiles = p->sp[j].stiles;
            b.ntiles = p->sp[j].sntiles;
            if ((st = launch_split_syn_dexp(b, s))) return st;
        }
        p->sp_dexp_valid = true;
    }
    return S2DWC_OK;
}

// Runs f(j, stream) for every scale: on the plan's per-scale streams forked
// from and joined back to `s`, or all on `s` in timing mode.
template <typename F>
int for_scales(s2dwc_plan *p, cudaStream_t s, F &&f)
{
    int st;
    if (p->timing) {
        for (int j = 0; j <= p->J; j++)
            if ((st = f(j, s))) return st;
        return S2DWC_OK;
    }
    S2DW_CUDA_TRY(cudaEventRecord(p->ev_fork, s));
    for (int j = 0; j <= p->J; j++) {
        S2DW_CUDA_TRY(cudaStreamWaitEvent(p->streams[j], p->ev_fork, 0));
        if ((st = f(j, p->streams[j]))) return st;
        S2DW_CUDA_TRY(cudaEventRecord(p->ev_join[j], p->streams[j]));
    }
    for (int j = 0; j <= p->J; j++) S2DW_CUDA_TRY(cudaStreamWaitEvent(s, p->ev_join[j], 0));
    return S2DWC_OK;
}

// Split-form analysis of `nmaps` maps (flm, wav and scoeff of map k at
// k * B^2, k * wav_total and k * bl_scoeff^2): per group of up to 32 maps,
// every scale on its own stream runs the map digits, the tensor-core
// contraction into Tg of the whole group, then the beta and alpha transforms
// map by map.
int run_analysis_split(s2dwc_plan *p, int nmaps, double *d_wav, double2 *d_scoeff, const double2 *d_flm,
                       cudaStream_t s)
{
    int st;
    if ((st = split_prepare(p, nmaps, s))) return st;
    const int MAPS = split_maps_per_pass();
    const long long wtot = p->wav_off[p->J + 1], B2 = (long long)p->B * p->B;
    const long long bs2 = (long long)p->bl_scoeff * p->bl_scoeff;
    for (int g0 = 0; g0 < nmaps; g0 += MAPS) {
        const int nk = std::min(MAPS, nmaps - g0);
        st = for_scales(p, s, [&](int j, cudaStream_t sj) -> int {
            int st2;
            const int bl = p->bl[j];
            const auto &S = p->sp[j];
            FdigArgs fa{};
            fa.B = p->B;
            fa.bl = bl;
            fa.blo = p->blo[j];
            fa.c0 = S.c0;
            fa.nch = S.nch;
            fa.nmaps = nk;
            fa.flm = d_flm + g0 * B2;
            fa.fexp = p->sp_fexp + S.fexp_off;
            fa.fdig = p->sp_fdig + S.fdig_off;
            {
                KernelTimer kt(p, S2DWC_KIND_OTHER, sj);
                if ((st2 = launch_split_fdig(fa, sj))) return st2;
            }
            SplitArgs a{};
            a.B = p->B;
            a.Bp = p->Bp;
            a.N = p->N;
            a.NP = p->NP;
            a.bl = bl;
            a.blo = p->blo[j];
            a.c0 = S.c0;
            a.nch = S.nch;
            a.nmaps = nk;
            std::memcpy(a.nq, p->nq, sizeof(a.nq));
            a.Acoef = p->Acoef;
            a.Om = p->Om;
            a.Stm = p->Stm;
            a.Ste = p->Ste;
            a.G = p->Ga + p->ga_off[j];
            a.Gs = p->ga_stride[j];
            a.dexp = p->sp_dexp + S.dexp_off;
            a.fexp = p->sp_fexp + S.fexp_off;
            a.fdig = p->sp_fdig + S.fdig_off;
            a.Tg = p->sp_Tg + p->sp_cap * S.tg_off;
            a.ph = p->sp_ph;
            a.tiles = S.tiles;
            a.ntiles = S.ntiles;
            a.err = p->sp_err;
            a.wait_ns = p->sp_wait_ns;
            {
                KernelTimer kt(p, S2DWC_KIND_LWALK, sj);
                if ((st2 = launch_split(a, sj))) return st2;
            }
            for (int k = 0; k < nk; k++) {
                CztArgs ca{};
                ca.mode = p->ana_beta_mode[j];
                ca.bl = bl;
                ca.N = p->N;
                ca.NP = p->NP;
                std::memcpy(ca.nq, p->nq, sizeof(ca.nq));
                ca.rows = p->N * bl;
                ca.czt = p->czt[j][ca.mode];
                if ((st = plan_tw(p, ca.czt.M, &ca.tw))) return st;
                ca.in_c = p->sp_Tg + p->sp_cap * S.tg_off + (long long)k * p->N * bl * bl;
                ca.out_c = p->sp_Tb + S.tb_off;
                {
                    KernelTimer kt(p, S2DWC_KIND_ANA_BETA, sj);
                    if ((st2 = launch_czt(ca, sj))) return st2;
                }
                ca.mode = CZT_ANA_ALPHA;
                ca.czt = p->czt[j][CZT_ANA_ALPHA];
                if ((st = plan_tw(p, ca.czt.M, &ca.tw))) return st;
                ca.in_c = p->sp_Tb + S.tb_off;
                ca.out_c = nullptr;
                ca.out_r = d_wav + (g0 + k) * wtot + p->wav_off[j];
                {
                    KernelTimer kt(p, S2DWC_KIND_ANA_ALPHA, sj);
                    if ((st2 = launch_czt(ca, sj))) return st2;
                }
            }
            return S2DWC_OK;
        });
        if (st) return st;
        for (int k = 0; k < nk; k++) {
            KernelTimer kt(p, S2DWC_KIND_OTHER, s);
            if ((st = launch_scoeff_copy(d_scoeff ? d_scoeff + (g0 + k) * bs2 : nullptr, d_flm + (g0 + k) * B2, p->B,
                                         p->bl_scoeff, s)))
                return st;
        }
    }
    return S2DWC_OK;
}

// Split-form synthesis of `nmaps` maps (layouts as run_analysis_split): per
// group of up to 32 maps, every scale on its own stream runs the alpha and
// beta transforms map by map into a batch of V tables, their digits and the
// tensor-core contraction into per-map partial rows; then the scale sum of
// each map, scales in order.
int run_synthesis_split(s2dwc_plan *p, int nmaps, double2 *d_flm, const double *d_wav, const double2 *d_scoeff,
                        cudaStream_t s)
{
    int st;
    if ((st = split_prepare(p, nmaps, s))) return st;
    const int MAPS = split_maps_per_pass();
    const long long wtot = p->wav_off[p->J + 1], B2 = (long long)p->B * p->B;
    const long long bs2 = (long long)p->bl_scoeff * p->bl_scoeff;
    for (int g0 = 0; g0 < nmaps; g0 += MAPS) {
        const int nk = std::min(MAPS, nmaps - g0);
        st = for_scales(p, s, [&](int j, cudaStream_t sj) -> int {
            int st2;
            const int bl = p->bl[j];
            const auto &S = p->sp[j];
            for (int k = 0; k < nk; k++) {
                CztArgs ca{};
                ca.mode = CZT_SYN_ALPHA;
                ca.bl = bl;
                ca.N = p->N;
                ca.NP = p->NP;
                std::memcpy(ca.nq, p->nq, sizeof(ca.nq));
                ca.rows = p->N * bl;
                ca.czt = p->czt[j][CZT_SYN_ALPHA];
                if ((st = plan_tw(p, ca.czt.M, &ca.tw))) return st;
                ca.in_r = d_wav + (g0 + k) * wtot + p->wav_off[j];
                ca.out_c = p->sp_Tb + S.tb_off;
                ca.scale = (4.0 * (M_PI * M_PI) / (double)p->N) / (2.0 * bl - 1.0);
                {
                    KernelTimer kt(p, S2DWC_KIND_SYN_ALPHA, sj);
                    if ((st2 = launch_czt(ca, sj))) return st2;
                }
                ca.mode = p->syn_beta_mode[j];
                ca.rows = p->NP * bl;
                ca.czt = p->czt[j][ca.mode];
                if ((st = plan_tw(p, ca.czt.M, &ca.tw))) return st;
                ca.in_c = p->sp_Tb + S.tb_off;
                ca.in_r = nullptr;
                ca.out_c = p->sp_V2f + p->sp_cap * S.v2f_off + k * S.vstride;
                ca.out_stride = p->gs_stride[j];
                ca.wq = p->wq[j];
                {
                    KernelTimer kt(p, S2DWC_KIND_SYN_BETA, sj);
                    if ((st2 = launch_czt(ca, sj))) return st2;
                }
            }
            if (bl - p->blo[j] - 1 <= 0) return S2DWC_OK;
            VdigArgs va{};
            va.bl = bl;
            va.NP = p->NP;
            va.nch = S.snch;
            va.nmaps = nk;
            va.Vs = p->gs_stride[j];
            va.V2f = p->sp_V2f + p->sp_cap * S.v2f_off;
            va.vstride = S.vstride;
            va.vexp = p->sp_vexp + S.fexp_off;
            va.vdig = p->sp_vdig + S.vdig_off;
            {
                KernelTimer kt(p, S2DWC_KIND_OTHER, sj);
                if ((st2 = launch_split_vdig(va, sj))) return st2;
            }
            SplitSynArgs b{};
            b.B = p->B;
            b.Bp = p->Bp;
            b.N = p->N;
            b.NP = p->NP;
            b.bl = bl;
            b.blo = p->blo[j];
            b.nch = S.snch;
            b.nmaps = nk;
            b.Bcoef = p->Bcoef;
            b.Em = p->Em;
            b.Ee = p->Ee;
            b.G = p->Gsyn + p->gs_off[j];
            b.Gs = p->gs_stride[j];
            b.sexp = p->sp_sexp + S.sexp_off;
            b.vexp = p->sp_vexp + S.fexp_off;
            b.vdig = p->sp_vdig + S.vdig_off;
            b.part = p->sp_part + p->offP[j];
            b.pstride = p->sp_pstride;
            b.tiles = S.stiles;
            b.ntiles = S.sntiles;
            b.err = p->sp_err;
            b.wait_ns = p->sp_wait_ns;
            KernelTimer kt(p, S2DWC_KIND_MWALK, sj);
            return launch_split_syn(b, sj);
        });
        if (st) return st;
        for (int k = 0; k < nk; k++) {
            CombineArgs cb{};
            cb.B = p->B;
            cb.J = p->J;
            cb.bs = p->bl_scoeff;
            for (int j = 0; j <= p->J; j++) {
                cb.bl[j] = p->bl[j];
                cb.blo[j] = p->blo[j];
                cb.off[j] = p->offP[j];
            }
            cb.parts = p->sp_part + k * p->sp_pstride;
            cb.scoeff = d_scoeff ? d_scoeff + (g0 + k) * bs2 : nullptr;
            cb.Phi2 = p->Phi2;
            cb.flm = d_flm + (g0 + k) * B2;
            KernelTimer kt(p, S2DWC_KIND_OTHER, s);
            if ((st = launch_combine(cb, s))) return st;
        }
    }
    return S2DWC_OK;
}

}  // namespace

extern "C" {

const char *s2dwc_version(void) { return "s2dw-b200 0.1 (sm_100a, FP64)"; }

int s2dwc_init(void)
{
    S2DW_API_TRY
    S2DW_CUDA_TRY(cudaFree(nullptr));
    return S2DWC_OK;
    S2DW_API_CATCH
}

int s2dwc_finalize(void)
{
    S2DW_API_TRY
    std::lock_guard<std::mutex> g(g_cache_mu);
    g_cache.clear();
    noalloc_forget();
    return S2DWC_OK;
    S2DW_API_CATCH
}

const char *s2dwc_error_string(int code)
{
    static const char *txt[] = {
        "No error",
        "Attempt to initialise object that has already been initialised",
        "Object not initialised",
        "Object initialisation failed",
        "Memory allocation failed",
        "Arithmetic exception",
        "Arithmetic warning",
        "Warning: Sizes not in recommended range",
        "Invalid sizes",
        "Sizes not defined",
        "Arguments invalid",
        "Argument warning",
        "Exceeded number of steps limit whem computing quadrature",
        "Admissibility test failed (resolution of identity not satisfied)",
        "File IO error",
        "CUDA runtime error",
    };
    if (code < 0 || code > 15) return "Unknown error";
    return txt[code];
}

int s2dwc_plan_create(s2dwc_plan **plan, int B, int N, double alpha, int J, int form, int device)
{
    S2DW_API_TRY
    if (!plan) return set_error(S2DWC_ERROR_ARG_INVALID, "plan_create: null output");
    *plan = nullptr;
    int st = validate_sizes(B, N, alpha, J);
    if (st) return st;
    if (form != S2DWC_FORM_FP64 && form != S2DWC_FORM_SPLIT)
        return set_error(S2DWC_ERROR_ARG_INVALID, "unknown form %d", form);
    if (form == S2DWC_FORM_SPLIT && N > 8)
        return set_error(S2DWC_ERROR_SIZE_INVALID, "N=%d: the split form supports N <= 8", N);
    if (const long long lim = g_plan_mem_limit.load()) {
        // checked on the host before any device call
        long long need = 0;
        if ((st = s2dwc_plan_footprint(B, N, alpha, J, form, &need))) return st;
        if (need > lim)
            return set_error(S2DWC_ERROR_MEM_ALLOC_FAIL,
                             "plan B=%d N=%d J=%d needs %lld bytes of device memory, above the plan memory "
                             "limit of %lld", B, N, J, need, lim);
    }
    int ndev = 0;
    S2DW_CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev)
        return set_error(S2DWC_ERROR_ARG_INVALID, "device %d out of range (%d devices)", device, ndev);
    DeviceGuard dg(device);
    if (const char *fv = getenv("S2DW_FFT_VALUES")) set_fft_values(atoi(fv));
    {
        const char *l2 = getenv("S2DW_LARGE_2048");
        set_large_2048(l2 ? atoi(l2) != 0 : true);
        const char *pf = getenv("S2DW_PFA");
        set_pfa(pf ? atoi(pf) != 0 : true);
        const char *pt = getenv("S2DW_PFA2047_THREADS");
        set_pfa2047_threads(pt ? atoi(pt) : 128);
        const char *p3 = getenv("S2DW_PFA1023");
        set_pfa1023(p3 ? atoi(p3) != 0 : true);
        const char *p5 = getenv("S2DW_PFA511");
        set_pfa511(p5 ? atoi(p5) != 0 : true);
        const char *ps = getenv("S2DW_PFA_SMALL");
        set_pfa_small(ps ? atoi(ps) != 0 : true);
    }
    {
        const char *ap = getenv("S2DW_ALPHA_PREFETCH");
        set_alpha_prefetch(ap ? atoi(ap) != 0 : true);
    }
    {
        const char *lw = getenv("S2DW_LWALK_VARIANT"), *mw = getenv("S2DW_MWALK_VARIANT");
        // default synthesis kernel: two l per thread (4; N > 8 falls back to 0)
        set_walk_variants(lw ? atoi(lw) : 0, mw ? atoi(mw) : 4);
    }
    auto *p = new s2dwc_plan();
    p->B = B;
    p->N = N;
    p->J = J;
    p->alpha = alpha;
    p->form = form;
    p->device = device;
    st = plan_build(p);
    if (st) {
        delete p;
        return st;
    }
    *plan = p;
    return S2DWC_OK;
    S2DW_API_CATCH
}

int s2dwc_plan_footprint(int B, int N, double alpha, int J, int form, long long *bytes)
{
    S2DW_API_TRY
    if (!bytes) return set_error(S2DWC_ERROR_ARG_INVALID, "plan_footprint: null output");
    *bytes = 0;
    int st = validate_sizes(B, N, alpha, J);
    if (st) return st;
    if (form != S2DWC_FORM_FP64 && form != S2DWC_FORM_SPLIT)
        return set_error(S2DWC_ERROR_ARG_INVALID, "unknown form %d", form);
    s2dwc_plan p;
    p.dry = true;
    p.B = B;
    p.N = N;
    p.J = J;
    p.alpha = alpha;
    p.form = form;
    if ((st = plan_build(&p))) return st;
    *bytes = p.ws_bytes;
    return S2DWC_OK;
    S2DW_API_CATCH
}

int s2dwc_set_plan_memory_limit(long long bytes)
{
    if (bytes < 0) return set_error(S2DWC_ERROR_ARG_INVALID, "plan memory limit %lld is negative", bytes);
    g_plan_mem_limit.store(bytes);
    return S2DWC_OK;
}

int s2dwc_plan_destroy(s2dwc_plan *plan)
{
    S2DW_API_TRY
    delete plan;
    return S2DWC_OK;
    S2DW_API_CATCH
}

int s2dwc_plan_set_tables(s2dwc_plan *p, const double *K_gamma, const double *Phi2, const double *Slm_,
                          int bl_scoeff)
{
    S2DW_API_TRY
    if (!p || !K_gamma || !Slm_) return set_error(S2DWC_ERROR_ARG_INVALID, "set_tables: null pointer");
    const int B = p->B, N = p->N, J = p->J, NP = p->NP;
    if (bl_scoeff < 0 || bl_scoeff > B)
        return set_error(S2DWC_ERROR_SIZE_INVALID, "bl_scoeff=%d outside [0,B]", bl_scoeff);
    const std::complex<double> *S = reinterpret_cast<const std::complex<double> *>(Slm_);
    // The kernels factor S(l,n) = eta (a(l,n) + i b(l,n)) with eta = 1 (N odd)
    // or i (N even) and a, b real.  s2dw_core_init_directionality produces
    // b = 0 (s2dw_core_mod.f90:240-245); any other Slm (b != 0 somewhere)
    // runs the contractions a second time with the tables of b.  Entries
    // with N+n even are never used.
    const bool even = (N % 2 == 0);
    std::vector<double> sa((size_t)B * NP), sb((size_t)B * NP);
    bool general = false;
    for (int q = 0; q < NP; q++)
        for (int l = 0; l < B; l++) {
            const std::complex<double> v = S[l + (size_t)B * p->nq[q]];
            // S / eta: eta = i divides as (x + i y) / i = y - i x
            sa[(size_t)l * NP + q] = even ? v.imag() : v.real();
            sb[(size_t)l * NP + q] = even ? -v.real() : v.imag();
            if (sb[(size_t)l * NP + q] != 0.0) general = true;
        }
    auto factors = [&](const std::vector<double> &s, std::vector<double> &kA, std::vector<double> &kS) {
        kA.assign((size_t)(J + 1) * B * NP, 0.0);
        kS.assign((size_t)(J + 1) * B * NP, 0.0);
        const double c8 = 8.0 * (M_PI * M_PI);
        for (int j = 0; j <= J; j++)
            for (int l = 0; l < B; l++) {
                const double K = K_gamma[j + (size_t)(J + 1) * l];
                for (int q = 0; q < NP; q++) {
                    const int n = p->nq[q];
                    const double sv = s[(size_t)l * NP + q];
                    kA[((size_t)j * B + l) * NP + q] = K * sv;
                    // (2l+1)/(8 pi^2) (1 or 2) K S i^{-n} with the eta i^{-n}
                    // phase reduced to the real sign (-1)^floor(n/2)
                    const double sig = ((n / 2) & 1) ? -1.0 : 1.0;
                    kS[((size_t)j * B + l) * NP + q] =
                        ((double)(2 * l + 1) / c8) * (n == 0 ? 1.0 : 2.0) * K * sv * sig;
                }
            }
    };
    std::vector<double> kA, kS;
    factors(sa, kA, kS);
    DeviceGuard dg(p->device);
    if (general && !p->Ga_b) {
        int st;
        if ((st = dev_alloc(p, &p->kappaA_b, (size_t)(J + 1) * B * NP)) ||
            (st = dev_alloc(p, &p->kappaS_b, (size_t)(J + 1) * B * NP)) ||
            (st = dev_alloc(p, &p->Ga_b, (size_t)std::max(1LL, p->ga_total))) ||
            (st = dev_alloc(p, &p->Gsyn_b, (size_t)std::max(1LL, p->gs_total))) ||
            (p->GsT && (st = dev_alloc(p, &p->GsT_b, (size_t)std::max(1LL, p->gt_total)))))
            return st;
    }
    if (general) {
        std::vector<double> kAb, kSb;
        factors(sb, kAb, kSb);
        S2DW_CUDA_TRY(cudaMemcpy(p->kappaA_b, kAb.data(), kAb.size() * sizeof(double), cudaMemcpyHostToDevice));
        S2DW_CUDA_TRY(cudaMemcpy(p->kappaS_b, kSb.data(), kSb.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    S2DW_CUDA_TRY(cudaMemcpy(p->kappaA, kA.data(), kA.size() * sizeof(double), cudaMemcpyHostToDevice));
    S2DW_CUDA_TRY(cudaMemcpy(p->kappaS, kS.data(), kS.size() * sizeof(double), cudaMemcpyHostToDevice));
    if (Phi2)
        S2DW_CUDA_TRY(cudaMemcpy(p->Phi2, Phi2, (size_t)B * sizeof(double), cudaMemcpyHostToDevice));
    else
        S2DW_CUDA_TRY(cudaMemset(p->Phi2, 0, (size_t)B * sizeof(double)));
    for (int j = 0; j <= J; j++) {
        GprepArgs g{};
        g.B = B;
        g.Bp = p->Bp;
        g.NP = NP;
        g.bl = p->bl[j];
        g.blo = p->blo[j];
        std::memcpy(g.nq, p->nq, sizeof(g.nq));
        g.H = p->H;
        g.hn = p->hn;
        g.T = p->Om;
        g.kappa = p->kappaA + (size_t)j * B * NP;
        g.stride = p->ga_stride[j];
        g.out = p->Ga + p->ga_off[j];
        int st = launch_gprep(g, 0);
        if (st) return st;
        g.T = p->Gam;
        g.kappa = p->kappaS + (size_t)j * B * NP;
        g.stride = p->gs_stride[j];
        g.out = p->Gsyn + p->gs_off[j];
        if ((st = launch_gprep(g, 0))) return st;
        if (general) {
            g.T = p->Om;
            g.kappa = p->kappaA_b + (size_t)j * B * NP;
            g.stride = p->ga_stride[j];
            g.out = p->Ga_b + p->ga_off[j];
            if ((st = launch_gprep(g, 0))) return st;
            g.T = p->Gam;
            g.kappa = p->kappaS_b + (size_t)j * B * NP;
            g.stride = p->gs_stride[j];
            g.out = p->Gsyn_b + p->gs_off[j];
            if ((st = launch_gprep(g, 0))) return st;
        }
        if (p->GsT) {
            GsTArgs t{};
            t.Bp = p->Bp;
            t.NP = NP;
            t.bl = p->bl[j];
            t.blo = p->blo[j];
            t.Gs = p->gs_stride[j];
            t.Ts = p->gt_ld[j];
            t.rows = (p->bl[j] + 7) / 8 * 8;
            t.G = p->Gsyn + p->gs_off[j];
            t.Bcoef = p->Bcoef;
            t.out = p->GsT + p->gt_off[j];
            if ((st = launch_gsyn_t(t, 0))) return st;
            if (general) {
                t.G = p->Gsyn_b + p->gs_off[j];
                t.out = p->GsT_b + p->gt_off[j];
                if ((st = launch_gsyn_t(t, 0))) return st;
            }
        }
    }
    S2DW_CUDA_TRY(cudaDeviceSynchronize());
    p->bl_scoeff = bl_scoeff;
    p->slm_general = general;
    p->tables_set = true;
    p->sp_dexp_valid = false;
    return S2DWC_OK;
    S2DW_API_CATCH
}

int s2dwc_plan_wav_offsets(const s2dwc_plan *p, long long *offsets)
{
    S2DW_API_TRY
    if (!p || !offsets) return set_error(S2DWC_ERROR_ARG_INVALID, "wav_offsets: null pointer");
    for (int j = 0; j <= p->J + 1; j++) offsets[j] = p->wav_off[j];
    return S2DWC_OK;
    S2DW_API_CATCH
}

long long s2dwc_plan_workspace_bytes(const s2dwc_plan *p) { return p ? p->ws_bytes : 0; }

int s2dwc_plan_launch_count(const s2dwc_plan *p, int *analysis, int *synthesis)
{
    S2DW_API_TRY
    if (!p) return set_error(S2DWC_ERROR_ARG_INVALID, "launch_count: null plan");
    // a general Slm runs each contraction twice
    const int g = p->slm_general ? 2 : 1;
    if (analysis) *analysis = (2 + g) * (p->J + 1) + 2;
    int ns = 1;
    for (int j = 0; j <= p->J; j++) ns += 2 + ((p->bl[j] - p->blo[j] - 1) > 0 ? g : 0);
    if (synthesis) *synthesis = ns;
    return S2DWC_OK;
    S2DW_API_CATCH
}

int s2dwc_plan_set_timing(s2dwc_plan *p, int enable)
{
    S2DW_API_TRY
    if (!p) return set_error(S2DWC_ERROR_ARG_INVALID, "set_timing: null plan");
    p->timing = enable != 0;
    return S2DWC_OK;
    S2DW_API_CATCH
}

int s2dwc_plan_timing(s2dwc_plan *p, int kind, long long *launches, double *total_ms)
{
    S2DW_API_TRY
    if (!p || kind < 0 || kind >= S2DWC_KIND_COUNT)
        return set_error(S2DWC_ERROR_ARG_INVALID, "timing: bad plan or kind %d", kind);
    DeviceGuard dg(p->device);
    for (auto &t : p->tev) {
        float ms = 0.f;
        S2DW_CUDA_TRY(cudaEventSynchronize(std::get<2>(t)));
        S2DW_CUDA_TRY(cudaEventElapsedTime(&ms, std::get<1>(t), std::get<2>(t)));
        p->t_ms[std::get<0>(t)] += ms;
        p->t_n[std::get<0>(t)] += 1;
        cudaEventDestroy(std::get<1>(t));
        cudaEventDestroy(std::get<2>(t));
    }
    p->tev.clear();
    if (launches) *launches = p->t_n[kind];
    if (total_ms) *total_ms = p->t_ms[kind];
    return S2DWC_OK;
    S2DW_API_CATCH
}

int s2dwc_plan_timing_reset(s2dwc_plan *p)
{
    S2DW_API_TRY
    if (!p) return set_error(S2DWC_ERROR_ARG_INVALID, "timing_reset: null plan");
    long long n;
    double ms;
    int st = s2dwc_plan_timing(p, 0, &n, &ms);
    for (int k = 0; k < S2DWC_KIND_COUNT; k++) {
        p->t_ms[k] = 0.0;
        p->t_n[k] = 0;
    }
    return st;
    S2DW_API_CATCH
}

int s2dwc_plan_analysis(s2dwc_plan *p, double *d_wav, double *d_scoeff, const double *d_flm, void *stream)
{
    S2DW_API_TRY
    if (!p || !d_wav || !d_flm || (!d_scoeff && p->bl_scoeff > 0))
        return set_error(S2DWC_ERROR_ARG_INVALID, "plan_analysis: null pointer");
    if (!p->tables_set) return set_error(S2DWC_ERROR_NOT_INIT, "plan_analysis: tables not set");
    DeviceGuard dg(p->device);
    if (p->form == S2DWC_FORM_SPLIT)
        return run_analysis_split(p, 1, d_wav, reinterpret_cast<double2 *>(d_scoeff),
                                  reinterpret_cast<const double2 *>(d_flm), (cudaStream_t)stream);
    return run_analysis(p, d_wav, reinterpret_cast<double2 *>(d_scoeff),
                        reinterpret_cast<const double2 *>(d_flm), (cudaStream_t)stream);
    S2DW_API_CATCH
}

int s2dwc_plan_analysis_batch(s2dwc_plan *p, int nmaps, double *d_wav, double *d_scoeff, const double *d_flm,
                              void *stream)
{
    S2DW_API_TRY
    if (!p || !d_wav || !d_flm || (!d_scoeff && p->bl_scoeff > 0))
        return set_error(S2DWC_ERROR_ARG_INVALID, "plan_analysis_batch: null pointer");
    if (nmaps < 0) return set_error(S2DWC_ERROR_ARG_INVALID, "plan_analysis_batch: nmaps=%d", nmaps);
    if (!p->tables_set) return set_error(S2DWC_ERROR_NOT_INIT, "plan_analysis_batch: tables not set");
    DeviceGuard dg(p->device);
    cudaStream_t s = (cudaStream_t)stream;
    if (p->form == S2DWC_FORM_SPLIT && nmaps >= p->sp_min_batch)
        return run_analysis_split(p, nmaps, d_wav, reinterpret_cast<double2 *>(d_scoeff),
                                  reinterpret_cast<const double2 *>(d_flm), s);
    const long long wtot = p->wav_off[p->J + 1], B2 = (long long)p->B * p->B;
    const long long bs2 = (long long)p->bl_scoeff * p->bl_scoeff;
    for (int k = 0; k < nmaps; k++) {
        int st = run_analysis(p, d_wav + k * wtot, d_scoeff ? reinterpret_cast<double2 *>(d_scoeff) + k * bs2 : nullptr,
                              reinterpret_cast<const double2 *>(d_flm) + k * B2, s);
        if (st) return st;
    }
    return S2DWC_OK;
    S2DW_API_CATCH
}

int s2dwc_plan_synthesis_batch(s2dwc_plan *p, int nmaps, double *d_flm, const double *d_wav, const double *d_scoeff,
                               void *stream)
{
    S2DW_API_TRY
    if (!p || !d_wav || !d_flm || (!d_scoeff && p->bl_scoeff > 0))
        return set_error(S2DWC_ERROR_ARG_INVALID, "plan_synthesis_batch: null pointer");
    if (nmaps < 0) return set_error(S2DWC_ERROR_ARG_INVALID, "plan_synthesis_batch: nmaps=%d", nmaps);
    if (!p->tables_set) return set_error(S2DWC_ERROR_NOT_INIT, "plan_synthesis_batch: tables not set");
    DeviceGuard dg(p->device);
    if (p->form == S2DWC_FORM_SPLIT && nmaps >= p->sp_min_batch)
        return run_synthesis_split(p, nmaps, reinterpret_cast<double2 *>(d_flm), d_wav,
                                   reinterpret_cast<const double2 *>(d_scoeff), (cudaStream_t)stream);
    const long long wtot = p->wav_off[p->J + 1], B2 = (long long)p->B * p->B;
    const long long bs2 = (long long)p->bl_scoeff * p->bl_scoeff;
    for (int k = 0; k < nmaps; k++) {
        int st = run_synthesis(p, reinterpret_cast<double2 *>(d_flm) + k * B2, d_wav + k * wtot,
                               d_scoeff ? reinterpret_cast<const double2 *>(d_scoeff) + k * bs2 : nullptr,
                               (cudaStream_t)stream);
        if (st) return st;
    }
    return S2DWC_OK;
    S2DW_API_CATCH
}

int s2dwc_plan_stat_moments(s2dwc_plan *p, int nmaps, const double *d_wav, const double *d_mask, double *d_moments,
                            void *stream)
{
    S2DW_API_TRY
    if (!p || !d_wav || !d_moments) return set_error(S2DWC_ERROR_ARG_INVALID, "plan_stat_moments: null pointer");
    if (nmaps < 0) return set_error(S2DWC_ERROR_ARG_INVALID, "plan_stat_moments: nmaps=%d", nmaps);
    DeviceGuard dg(p->device);
    constexpr int G = 32;
    int st;
    if (!p->st_part) {
        const size_t ny = (size_t)G * (p->J + 1);
        if ((st = dev_alloc(p, &p->st_part, ny * STAT_P * 6)) || (st = dev_alloc(p, &p->st_mean, ny * 2)) ||
            (st = dev_alloc(p, &p->st_flags, ny)))
            return st;
    }
    const long long wtot = p->wav_off[p->J + 1];
    for (int g0 = 0; g0 < nmaps; g0 += G) {
        StatArgs a{};
        a.J = p->J;
        a.nmaps = std::min(G, nmaps - g0);
        a.wtot = wtot;
        for (int j = 0; j <= p->J + 1; j++) a.off[j] = p->wav_off[j];
        a.wav = d_wav + (size_t)g0 * wtot;
        a.mask = d_mask;
        a.part = p->st_part;
        a.mean_nj = p->st_mean;
        a.out = d_moments + (size_t)g0 * (p->J + 1) * 6;
        a.flags = p->st_flags;
        if ((st = launch_stat_moments(a, (cudaStream_t)stream))) return st;
    }
    return S2DWC_OK;
    S2DW_API_CATCH
}

int s2dwc_stat_moments(double *const *wav_scales, int J, int B, int N, double alpha, double *mean, double *var,
                       double *skew, double *kur, const double *const *mask_scales, double *five, double *six)
{
    S2DW_API_TRY
    if (!wav_scales || !mean || !var || !skew || !kur)
        return set_error(S2DWC_ERROR_ARG_INVALID, "stat_moments: null pointer");
    if (B < 2 || N < 1 || J < 0 || J > S2DW_JMAX || !(alpha > 1.0))
        return set_error(S2DWC_ERROR_SIZE_INVALID, "stat_moments: B=%d N=%d J=%d alpha=%g", B, N, J, alpha);
    for (int j = 0; j <= J; j++)
        if (!wav_scales[j] || (mask_scales && !mask_scales[j]))
            return set_error(S2DWC_ERROR_ARG_INVALID, "stat_moments: scale %d is null", j);
    StatArgs a{};
    a.J = J;
    a.nmaps = 1;
    a.off[0] = 0;
    for (int j = 0; j <= J; j++) {
        int hi, lo;
        band_limits(j, B, alpha, &hi, &lo);
        a.off[j + 1] = a.off[j] + (long long)(2 * hi - 1) * (2 * hi) * N;
    }
    a.wtot = a.off[J + 1];
    const size_t ny = (size_t)J + 1;
    // one device block for everything this call needs, freed before return
    const size_t nw = (size_t)a.wtot, nm = mask_scales ? nw : 0;
    const size_t bytes = 8 * (nw + nm + ny * STAT_P * 6 + ny * 2 + ny * 6) + 4 * ny + 256;
    char *blk = nullptr;
    cudaError_t e = cudaMalloc(&blk, bytes);
    if (e != cudaSuccess)
        return set_error(S2DWC_ERROR_MEM_ALLOC_FAIL, "stat_moments: cudaMalloc of %zu bytes failed: %s", bytes,
                         cudaGetErrorString(e));
    std::unique_ptr<char, void (*)(char *)> guard(blk, [](char *q) { cudaFree(q); });
    double *dw = reinterpret_cast<double *>(blk), *dm = dw + nw, *dpart = dm + nm, *dmean = dpart + ny * STAT_P * 6,
           *dout = dmean + ny * 2;
    int *dflags = reinterpret_cast<int *>(dout + ny * 6);
    for (int j = 0; j <= J; j++) {
        const size_t n = (size_t)(a.off[j + 1] - a.off[j]);
        S2DW_CUDA_TRY(cudaMemcpy(dw + a.off[j], wav_scales[j], 8 * n, cudaMemcpyHostToDevice));
        if (mask_scales) S2DW_CUDA_TRY(cudaMemcpy(dm + a.off[j], mask_scales[j], 8 * n, cudaMemcpyHostToDevice));
    }
    a.wav = dw;
    a.mask = mask_scales ? dm : nullptr;
    a.part = dpart;
    a.mean_nj = dmean;
    a.out = dout;
    a.flags = dflags;
    int st = launch_stat_moments(a, 0);
    if (st) return st;
    std::vector<double> out(ny * 6);
    std::vector<int> flags(ny);
    S2DW_CUDA_TRY(cudaMemcpy(out.data(), dout, 8 * out.size(), cudaMemcpyDeviceToHost));
    S2DW_CUDA_TRY(cudaMemcpy(flags.data(), dflags, 4 * flags.size(), cudaMemcpyDeviceToHost));
    // the reference masks its input in place (s2dw_stat_mod.f90:121-125)
    if (mask_scales)
        for (int j = 0; j <= J; j++) {
            const long long n = a.off[j + 1] - a.off[j];
            double *w = wav_scales[j];
            const double *m = mask_scales[j];
#pragma omp parallel for
            for (long long i = 0; i < n; i++) w[i] *= m[i];
        }
    int status = S2DWC_OK;
    for (int j = 0; j <= J; j++) {
        if (flags[j] == 2)
            return set_error(S2DWC_ERROR_SIZE_INVALID, "stat_moments: scale %d has fewer than two samples", j);
        mean[j] = out[6 * j];
        var[j] = out[6 * j + 1];
        skew[j] = out[6 * j + 2];
        kur[j] = out[6 * j + 3];
        if (five) five[j] = out[6 * j + 4];
        if (five && six) six[j] = out[6 * j + 5];
        if (flags[j] == 1)
            status = set_error(S2DWC_ERROR_ARTH_WARNING,
                               "stat_moments: scale %d has zero variance; its higher moments are set to zero", j);
    }
    return status;
    S2DW_API_CATCH
}

int s2dwc_plan_reserve(s2dwc_plan *p, int nmaps, void *stream)
{
    S2DW_API_TRY
    if (!p) return set_error(S2DWC_ERROR_ARG_INVALID, "plan_reserve: null plan");
    if (nmaps < 0) return set_error(S2DWC_ERROR_ARG_INVALID, "plan_reserve: nmaps=%d", nmaps);
    if (p->form != S2DWC_FORM_SPLIT) return S2DWC_OK;
    if (!p->tables_set) return set_error(S2DWC_ERROR_NOT_INIT, "plan_reserve: tables not set");
    DeviceGuard dg(p->device);
    std::lock_guard<std::mutex> g(p->mu);
    return split_prepare(p, nmaps, (cudaStream_t)stream);
    S2DW_API_CATCH
}

int s2dwc_plan_check(s2dwc_plan *p)
{
    S2DW_API_TRY
    if (!p) return set_error(S2DWC_ERROR_ARG_INVALID, "plan_check: null plan");
    if (!p->sp_err) return S2DWC_OK;
    DeviceGuard dg(p->device);
    int h = 0;
    S2DW_CUDA_TRY(cudaMemcpy(&h, p->sp_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) {
        // reported once: the flag is cleared so that later calls start clean
        S2DW_CUDA_TRY(cudaMemset(p->sp_err, 0, sizeof(int)));
        return set_error(S2DWC_ERROR_CUDA, "a split-form kernel gave up waiting for its tensor-core pipeline");
    }
    return S2DWC_OK;
    S2DW_API_CATCH
}

int s2dwc_plan_set_priority(s2dwc_plan *p, int priority)
{
    S2DW_API_TRY
    if (!p) return set_error(S2DWC_ERROR_ARG_INVALID, "plan_set_priority: null plan");
    std::lock_guard<std::mutex> g(p->mu);
    DeviceGuard dg(p->device);
    int least = 0, greatest = 0;
    S2DW_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    const int prio = std::min(least, std::max(greatest, priority));
    for (auto &st : p->streams) {
        S2DW_CUDA_TRY(cudaStreamSynchronize(st));
        S2DW_CUDA_TRY(cudaStreamDestroy(st));
        st = nullptr;
        S2DW_CUDA_TRY(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, prio));
    }
    return S2DWC_OK;
    S2DW_API_CATCH
}

int s2dwc_plan_set_split_min_batch(s2dwc_plan *p, int nmaps)
{
    S2DW_API_TRY
    if (!p) return set_error(S2DWC_ERROR_ARG_INVALID, "plan_set_split_min_batch: null plan");
    if (nmaps < 1) return set_error(S2DWC_ERROR_ARG_INVALID, "plan_set_split_min_batch: nmaps=%d", nmaps);
    p->sp_min_batch = nmaps;
    return S2DWC_OK;
    S2DW_API_CATCH
}

int s2dwc_plan_set_wait_limit(s2dwc_plan *p, long long ns)
{
    S2DW_API_TRY
    if (!p) return set_error(S2DWC_ERROR_ARG_INVALID, "plan_set_wait_limit: null plan");
    if (ns < 0) return set_error(S2DWC_ERROR_ARG_INVALID, "plan_set_wait_limit: negative limit %lld", ns);
    p->sp_wait_ns = ns == 0 ? 0ull : (unsigned long long)ns;
    return S2DWC_OK;
    S2DW_API_CATCH
}

int s2dwc_plan_synthesis(s2dwc_plan *p, double *d_flm, const double *d_wav, const double *d_scoeff, void *stream)
{
    S2DW_API_TRY
    if (!p || !d_wav || !d_flm || (!d_scoeff && p->bl_scoeff > 0))
        return set_error(S2DWC_ERROR_ARG_INVALID, "plan_synthesis: null pointer");
    if (!p->tables_set) return set_error(S2DWC_ERROR_NOT_INIT, "plan_synthesis: tables not set");
    DeviceGuard dg(p->device);
    if (p->form == S2DWC_FORM_SPLIT)
        return run_synthesis_split(p, 1, reinterpret_cast<double2 *>(d_flm), d_wav,
                                   reinterpret_cast<const double2 *>(d_scoeff), (cudaStream_t)stream);
    return run_synthesis(p, reinterpret_cast<double2 *>(d_flm), d_wav,
                         reinterpret_cast<const double2 *>(d_scoeff), (cudaStream_t)stream);
    S2DW_API_CATCH
}

int s2dwc_plan_analysis_noalloc(const s2dwc_plan *p, double *d_wav, double *d_scoeff, const double *d_flm,
                                void *stream)
{
    S2DW_API_TRY
    if (!p || !d_wav || !d_flm || (!d_scoeff && p->bl_scoeff > 0))
        return set_error(S2DWC_ERROR_ARG_INVALID, "plan_analysis_noalloc: null pointer");
    if (!p->tables_set) return set_error(S2DWC_ERROR_NOT_INIT, "plan_analysis_noalloc: tables not set");
    if (p->form != S2DWC_FORM_FP64)
        return set_error(S2DWC_ERROR_ARG_INVALID,
                         "plan_analysis_noalloc runs the FP64 form only; create the plan with S2DWC_FORM_FP64");
    const SerialLayout L = serial_layout(p);
    if (L.bytes > S2DWC_NOALLOC_SCRATCH_BYTES)
        return set_error(S2DWC_ERROR_SIZE_INVALID,
                         "plan_analysis_noalloc: B=%d N=%d needs %lld bytes of scratch, more than the "
                         "%lld-byte static scratch (it holds B<=256 with N<=10, or B<=512 with N<=2); "
                         "use s2dwc_plan_analysis",
                         p->B, p->N, L.bytes, (long long)S2DWC_NOALLOC_SCRATCH_BYTES);
    DeviceGuard dg(p->device);
    void *ws = nullptr;
    int st = noalloc_scratch(p->device, &ws);
    if (st) return st;
    return run_analysis_serial(p, static_cast<unsigned char *>(ws), d_wav, reinterpret_cast<double2 *>(d_scoeff),
                               reinterpret_cast<const double2 *>(d_flm), (cudaStream_t)stream);
    S2DW_API_CATCH
}

// ---------------------------------------------------------------------------
// Host-buffer entry points
// ---------------------------------------------------------------------------

// Device buffers of the host-buffer entry points, owned by the plan and
// reused across calls (the plan mutex serialises their use).
struct HostCallBuffers {
    double *wav = nullptr;
    double2 *flm = nullptr, *sc = nullptr;
};

// Folds the caller's tables into the cached plan unless they equal, byte for
// byte, the ones folded last: callers pass the same K_gamma and Slm on every
// call, and refolding them costs 2(J+1) table kernels and a device
// synchronisation per call.  Phi2 (synthesis only) is compared and uploaded
// on its own; the analysis passes none and leaves the plan's copy as is.
static int host_fold_tables(s2dwc_plan *p, const double *K_gamma, const double *Phi2, const double *Slm,
                            int bl_scoeff)
{
    const size_t nK = (size_t)(p->J + 1) * p->B, nS = 2 * (size_t)p->B * p->N, nP = (size_t)p->B;
    const bool same = p->tables_set && p->hc_bls == bl_scoeff && p->hc_K.size() == nK && p->hc_S.size() == nS &&
                      std::memcmp(p->hc_K.data(), K_gamma, nK * sizeof(double)) == 0 &&
                      std::memcmp(p->hc_S.data(), Slm, nS * sizeof(double)) == 0;
    if (!same) {
        p->hc_K.clear();
        p->hc_S.clear();
        p->hc_Phi2.clear();
        int st = s2dwc_plan_set_tables(p, K_gamma, Phi2, Slm, bl_scoeff);
        if (st) return st;
        p->hc_K.assign(K_gamma, K_gamma + nK);
        p->hc_S.assign(Slm, Slm + nS);
        if (Phi2) p->hc_Phi2.assign(Phi2, Phi2 + nP);
        p->hc_bls = bl_scoeff;
        return S2DWC_OK;
    }
    if (Phi2 && (p->hc_Phi2.size() != nP || std::memcmp(p->hc_Phi2.data(), Phi2, nP * sizeof(double)) != 0)) {
        DeviceGuard dg(p->device);
        p->hc_Phi2.clear();
        S2DW_CUDA_TRY(cudaMemcpy(p->Phi2, Phi2, nP * sizeof(double), cudaMemcpyHostToDevice));
        p->hc_Phi2.assign(Phi2, Phi2 + nP);
    }
    return S2DWC_OK;
}

// Looks up the cached plan of (B, N, alpha, J), takes its lock for the rest
// of the call, folds the tables and returns the plan's host-call buffers.
static int host_prepare(int B, int N, double alpha, int J, int bl_scoeff, const double *K_gamma,
                        const double *Phi2, const double *Slm, s2dwc_plan **pp, HostCallBuffers &hb,
                        std::unique_lock<std::mutex> &lk)
{
    int st = validate_sizes(B, N, alpha, J);
    if (st) return st;
    if ((st = get_cached_plan(B, N, alpha, J, pp))) return st;
    s2dwc_plan *p = *pp;
    lk = std::unique_lock<std::mutex>(p->mu);
    if ((st = host_fold_tables(p, K_gamma, Phi2, Slm, bl_scoeff))) return st;
    DeviceGuard dg(p->device);
    if (!p->copy_stream) {
        p->ev_done.assign(J + 1, nullptr);
        p->ev_copy.assign(J + 1, nullptr);
        for (int j = 0; j <= J; j++) {
            S2DW_CUDA_TRY(cudaEventCreateWithFlags(&p->ev_done[j], cudaEventDisableTiming));
            S2DW_CUDA_TRY(cudaEventCreateWithFlags(&p->ev_copy[j], cudaEventDisableTiming));
        }
        S2DW_CUDA_TRY(cudaEventCreateWithFlags(&p->ev_host, cudaEventDisableTiming));
        S2DW_CUDA_TRY(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking));
    }
    if (!p->hbWav) {
        if ((st = dev_alloc(p, &p->hbWav, (size_t)std::max(1LL, p->wav_off[J + 1]))) ||
            (st = dev_alloc(p, &p->hbFlm, (size_t)B * B)))
            return st;
    }
    if (p->hbSc_n < bl_scoeff * bl_scoeff || !p->hbSc) {
        if ((st = dev_alloc(p, &p->hbSc, (size_t)std::max(1, bl_scoeff * bl_scoeff)))) return st;
        p->hbSc_n = std::max(1, bl_scoeff * bl_scoeff);
    }
    hb.wav = p->hbWav;
    hb.flm = p->hbFlm;
    hb.sc = p->hbSc;
    return S2DWC_OK;
}

// Copies between pageable caller memory and the device through the plan's
// two page-locked staging buffers: the DMA of one chunk overlaps the host
// copy (OpenMP threads) of the other.  The driver's own pageable copies run
// at about a third of the page-locked rate, which made the host entry points
// three times slower for callers with ordinary (Fortran, numpy) arrays.
struct HostSeg {
    char *host;
    char *dev;
    size_t bytes;
};
constexpr size_t STAGE_BYTES = 32u << 20;

static void host_copy(char *dst, const char *src, size_t n)
{
    const long long blk = 1 << 20, nb = (long long)((n + blk - 1) / blk);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < nb; i++) {
        const size_t o = (size_t)(i * blk);
        std::memcpy(dst + o, src + o, std::min((size_t)blk, n - o));
    }
}

// A staged copy that can be run a segment at a time: the synthesis queues
// each scale's kernels as soon as that scale's chunks are on their way, and
// the analysis lets each segment's first chunk wait for its scale's kernels,
// so the host copies and the DMA overlap the other scales' kernels.
class StagedCopy {
  public:
    StagedCopy(s2dwc_plan *p, const std::vector<HostSeg> &segs, cudaStream_t s) : p_(p), s_(s)
    {
        for (const auto &g : segs) {
            for (size_t o = 0; o < g.bytes; o += STAGE_BYTES)
                ch_.push_back({g.host + o, g.dev + o, std::min(STAGE_BYTES, g.bytes - o)});
            seg_end_.push_back(ch_.size());
        }
    }
    // Allocates the staging buffers on first use and waits for an earlier
    // call's DMA on them.
    int start()
    {
        for (int i = 0; i < 2; i++) {
            if (!p_->stage[i]) {
                S2DW_CUDA_TRY(
                    cudaHostAlloc(reinterpret_cast<void **>(&p_->stage[i]), STAGE_BYTES, cudaHostAllocDefault));
                S2DW_CUDA_TRY(cudaEventCreateWithFlags(&p_->stage_ev[i], cudaEventDisableTiming));
                S2DW_CUDA_TRY(cudaEventRecord(p_->stage_ev[i], s_));
            }
            S2DW_CUDA_TRY(cudaEventSynchronize(p_->stage_ev[i]));
        }
        return S2DWC_OK;
    }
    // Host to device: queues every chunk of segments up to k (inclusive).
    int to_device_through(size_t k)
    {
        for (; next_ < seg_end_[k]; next_++) {
            const size_t i = next_;
            const int b = (int)(i & 1);
            if (i >= 2) S2DW_CUDA_TRY(cudaEventSynchronize(p_->stage_ev[b]));  // chunk i-2's DMA done
            host_copy(p_->stage[b], ch_[i].host, ch_[i].n);
            S2DW_CUDA_TRY(cudaMemcpyAsync(ch_[i].dev, p_->stage[b], ch_[i].n, cudaMemcpyHostToDevice, s_));
            S2DW_CUDA_TRY(cudaEventRecord(p_->stage_ev[b], s_));
        }
        return S2DWC_OK;
    }
    // Device to host, every segment; segment k's DMA first waits for wait[k]
    // (when given) and seg_done(k) runs on the host once segment k is in the
    // caller's memory.
    int to_host(const cudaEvent_t *wait = nullptr, const std::function<void(size_t)> &seg_done = nullptr)
    {
        size_t k = 0;  // segment of chunk i
        for (size_t i = 0; i < ch_.size(); i++) {
            while (seg_end_[k] <= i) k++;
            const int b = (int)(i & 1);
            if (wait && i == (k ? seg_end_[k - 1] : 0))  // segment k's first chunk
                S2DW_CUDA_TRY(cudaStreamWaitEvent(s_, wait[k], 0));
            S2DW_CUDA_TRY(cudaMemcpyAsync(p_->stage[b], ch_[i].dev, ch_[i].n, cudaMemcpyDeviceToHost, s_));
            S2DW_CUDA_TRY(cudaEventRecord(p_->stage_ev[b], s_));
            if (i >= 1) {  // the previous chunk, while this one's DMA runs
                if (int st = drain(i - 1, seg_done)) return st;
            }
        }
        if (!ch_.empty())
            if (int st = drain(ch_.size() - 1, seg_done)) return st;
        // segments without chunks (empty scales) are complete at once
        if (seg_done)
            for (size_t q = 0; q < seg_end_.size(); q++)
                if (seg_end_[q] == (q ? seg_end_[q - 1] : 0)) seg_done(q);
        return S2DWC_OK;
    }

  private:
    struct Chunk {
        char *host, *dev;
        size_t n;
    };
    int drain(size_t i, const std::function<void(size_t)> &seg_done)
    {
        const int b = (int)(i & 1);
        S2DW_CUDA_TRY(cudaEventSynchronize(p_->stage_ev[b]));
        host_copy(ch_[i].host, p_->stage[b], ch_[i].n);
        if (seg_done)
            for (size_t q = 0; q < seg_end_.size(); q++)
                if (seg_end_[q] == i + 1 && seg_end_[q] != (q ? seg_end_[q - 1] : 0)) seg_done(q);
        return S2DWC_OK;
    }
    s2dwc_plan *p_;
    cudaStream_t s_;
    std::vector<Chunk> ch_;
    std::vector<size_t> seg_end_;  // one past each segment's last chunk
    size_t next_ = 0;
};

// True when every pointer is page-locked host memory: then per-scale copies
// can be queued asynchronously on the scales' streams without blocking the
// host thread that queues the kernels.
static bool all_pinned(const void *const *ptrs, int n)
{
    for (int i = 0; i < n; i++) {
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, ptrs[i]) != cudaSuccess || at.type != cudaMemoryTypeHost) {
            cudaGetLastError();
            return false;
        }
    }
    return true;
}

static int analysis_host(double *wav_static, double *const *wav_scales, double *scoeff, const double *flm,
                         const double *K_gamma, const double *Slm, int J, int B, int N, int bl_scoeff,
                         double alpha)
{
    if (!flm || !K_gamma || !Slm || (!scoeff && bl_scoeff > 0) || (!wav_static && !wav_scales))
        return set_error(S2DWC_ERROR_ARG_INVALID, "analysis: null pointer");
    s2dwc_plan *p = nullptr;
    HostCallBuffers hb;
    std::unique_lock<std::mutex> lk;
    int st = host_prepare(B, N, alpha, J, bl_scoeff, K_gamma, nullptr, Slm, &p, hb, lk);
    if (st) return st;
    DeviceGuard dg(p->device);
    S2DW_CUDA_TRY(cudaMemcpy(hb.flm, flm, sizeof(double2) * (size_t)B * B, cudaMemcpyHostToDevice));
    // The scales' device-to-host copies overlap the other scales' kernels,
    // with the full-band scales run one after another.  Pinned per-scale
    // outputs: each copy follows its scale's kernels on the scale's stream.
    // Otherwise the staged copy (largest scale first) lets each scale's first
    // chunk wait for that scale's kernels.
    const bool pinned = wav_scales && all_pinned(reinterpret_cast<const void *const *>(wav_scales), J + 1);
    ScaleHook after = [&](int j, cudaStream_t sj) -> int {
        if (pinned)
            S2DW_CUDA_TRY(cudaMemcpyAsync(wav_scales[j], hb.wav + p->wav_off[j],
                                          sizeof(double) * (size_t)(p->wav_off[j + 1] - p->wav_off[j]),
                                          cudaMemcpyDeviceToHost, sj));
        else
            S2DW_CUDA_TRY(cudaEventRecord(p->ev_copy[j], sj));
        return S2DWC_OK;
    };
    if ((st = run_analysis(p, hb.wav, hb.sc, hb.flm, 0, after, true))) {
        // no copy into the caller's arrays may outlive the call
        for (int j = 0; j <= J; j++) cudaStreamSynchronize(p->streams[j]);
        return st;
    }
    if (!pinned) {
        std::unique_ptr<double[]> tmp;  // the static layout's per-scale blocks, uninitialised
        if (!wav_scales) tmp.reset(new double[std::max<long long>(p->wav_off[J + 1], 1)]);
        std::vector<HostSeg> segs;
        std::vector<cudaEvent_t> wait;
        for (int j = J; j >= 0; j--) {
            char *h = wav_scales ? reinterpret_cast<char *>(wav_scales[j])
                                 : reinterpret_cast<char *>(tmp.get() + p->wav_off[j]);
            segs.push_back({h, reinterpret_cast<char *>(hb.wav + p->wav_off[j]),
                            sizeof(double) * (size_t)(p->wav_off[j + 1] - p->wav_off[j])});
            wait.push_back(p->ev_copy[j]);
        }
        // scatter a scale into wav(0:J,0:2B-2,0:2B-1,0:N-1) once it is in the
        // host buffer; untouched outside each scale's region, as in
        // s2dw_core_mod.f90:509
        const size_t J1 = (size_t)J + 1, A = 2 * (size_t)B - 1, BB = 2 * (size_t)B;
        auto scatter = [&](size_t k) {
            const int j = J - (int)k, bl = p->bl[j], n = 2 * bl - 1;
            const double *src = tmp.get() + p->wav_off[j];
#pragma omp parallel for collapse(2)
            for (int g = 0; g < N; g++)
                for (int b = 0; b < 2 * bl; b++)
                    for (int a = 0; a < n; a++)
                        wav_static[j + J1 * (a + A * (b + BB * g))] = src[a + (size_t)n * (b + 2 * (size_t)bl * g)];
        };
        StagedCopy sc(p, segs, p->copy_stream);
        std::function<void(size_t)> seg_done;
        if (!wav_scales) seg_done = scatter;
        if ((st = sc.start()) || (st = sc.to_host(wait.data(), seg_done))) {
            cudaStreamSynchronize(p->copy_stream);
            return st;
        }
    }
    if (bl_scoeff > 0)
        S2DW_CUDA_TRY(cudaMemcpy(scoeff, hb.sc, sizeof(double2) * (size_t)bl_scoeff * bl_scoeff,
                                 cudaMemcpyDeviceToHost));
    S2DW_CUDA_TRY(cudaStreamSynchronize(0));
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

int s2dwc_analysis_flm2wav(double *wav, double *scoeff, const double *flm, const double *K_gamma,
                           const double *Slm, int J, int B, int N, int bl_scoeff, double alpha)
{
    S2DW_API_TRY
    if (!wav) return set_error(S2DWC_ERROR_ARG_INVALID, "analysis: null wav");
    return analysis_host(wav, nullptr, scoeff, flm, K_gamma, Slm, J, B, N, bl_scoeff, alpha);
    S2DW_API_CATCH
}

int s2dwc_analysis_flm2wav_dynamic(double *const *wav_scales, double *scoeff, const double *flm,
                                   const double *K_gamma, const double *Slm, int J, int B, int N,
                                   int bl_scoeff, double alpha)
{
    S2DW_API_TRY
    if (!wav_scales) return set_error(S2DWC_ERROR_ARG_INVALID, "analysis: null wav_scales");
    for (int j = 0; j <= J; j++)
        if (!wav_scales[j]) return set_error(S2DWC_ERROR_ARG_INVALID, "analysis: wav_scales[%d] is null", j);
    return analysis_host(nullptr, wav_scales, scoeff, flm, K_gamma, Slm, J, B, N, bl_scoeff, alpha);
    S2DW_API_CATCH
}

static int synthesis_host(double *flm, const double *wav_static, const double *const *wav_scales,
                          const double *scoeff, const double *K_gamma, const double *Phi2,
                          const double *Slm, int J, int B, int N, int bl_scoeff, double alpha)
{
    if (!flm || !K_gamma || !Phi2 || !Slm || (!scoeff && bl_scoeff > 0) || (!wav_static && !wav_scales))
        return set_error(S2DWC_ERROR_ARG_INVALID, "synthesis: null pointer");
    s2dwc_plan *p = nullptr;
    HostCallBuffers hb;
    std::unique_lock<std::mutex> lk;
    int st = host_prepare(B, N, alpha, J, bl_scoeff, K_gamma, Phi2, Slm, &p, hb, lk);
    if (st) return st;
    DeviceGuard dg(p->device);
    // One copy stream brings the scales in, the last (largest) first, and
    // each scale's kernels wait for their own copy only, so the largest
    // scales' kernels overlap the remaining copies and the kernels left after
    // the last copy are the small scales'.  Pinned per-scale inputs are
    // queued at once; otherwise each scale's staged chunks (gathered from the
    // static layout first, for that entry point) are queued just before the
    // scale's kernels.
    const bool pinned = wav_scales && all_pinned(reinterpret_cast<const void *const *>(wav_scales), J + 1);
    S2DW_CUDA_TRY(cudaEventRecord(p->ev_host, 0));
    S2DW_CUDA_TRY(cudaStreamWaitEvent(p->copy_stream, p->ev_host, 0));
    std::unique_ptr<double[]> tmp;  // the static layout's per-scale blocks
    if (!wav_scales) tmp.reset(new double[std::max<long long>(p->wav_off[J + 1], 1)]);
    std::vector<HostSeg> segs;
    for (int j = J; j >= 0; j--) {
        const size_t bytes = sizeof(double) * (size_t)(p->wav_off[j + 1] - p->wav_off[j]);
        if (pinned) {
            S2DW_CUDA_TRY(cudaMemcpyAsync(hb.wav + p->wav_off[j], wav_scales[j], bytes, cudaMemcpyHostToDevice,
                                          p->copy_stream));
            S2DW_CUDA_TRY(cudaEventRecord(p->ev_copy[j], p->copy_stream));
        } else {
            char *h = wav_scales ? const_cast<char *>(reinterpret_cast<const char *>(wav_scales[j]))
                                 : reinterpret_cast<char *>(tmp.get() + p->wav_off[j]);
            segs.push_back({h, reinterpret_cast<char *>(hb.wav + p->wav_off[j]), bytes});
        }
    }
    StagedCopy sc(p, segs, p->copy_stream);
    if (!pinned && (st = sc.start())) return st;
    if (bl_scoeff > 0)
        S2DW_CUDA_TRY(cudaMemcpy(hb.sc, scoeff, sizeof(double2) * (size_t)bl_scoeff * bl_scoeff,
                                 cudaMemcpyHostToDevice));
    const size_t J1 = (size_t)J + 1, A = 2 * (size_t)B - 1, BB = 2 * (size_t)B;
    ScaleHook copy_in = [&](int j, cudaStream_t sj) -> int {
        if (!pinned) {
            if (!wav_scales) {  // gather scale j from wav(0:J,0:2B-2,0:2B-1,0:N-1)
                const int bl = p->bl[j], n = 2 * bl - 1;
                double *dst = tmp.get() + p->wav_off[j];
#pragma omp parallel for collapse(2)
                for (int g = 0; g < N; g++)
                    for (int b = 0; b < 2 * bl; b++)
                        for (int a = 0; a < n; a++)
                            dst[a + (size_t)n * (b + 2 * (size_t)bl * g)] = wav_static[j + J1 * (a + A * (b + BB * g))];
            }
            if (int e = sc.to_device_through((size_t)(J - j))) return e;
            S2DW_CUDA_TRY(cudaEventRecord(p->ev_copy[j], p->copy_stream));
        }
        S2DW_CUDA_TRY(cudaStreamWaitEvent(sj, p->ev_copy[j], 0));
        return S2DWC_OK;
    };
    if ((st = run_synthesis(p, hb.flm, hb.wav, hb.sc, 0, copy_in, !pinned))) {
        cudaStreamSynchronize(p->copy_stream);  // no read of the caller's arrays outlives the call
        return st;
    }
    S2DW_CUDA_TRY(cudaMemcpy(flm, hb.flm, sizeof(double2) * (size_t)B * B, cudaMemcpyDeviceToHost));
    return S2DWC_OK;
}

int s2dwc_synthesis_wav2flm(double *flm, const double *wav, const double *scoeff, const double *K_gamma,
                            const double *Phi2, const double *Slm, int J, int B, int N, int bl_scoeff,
                            double alpha)
{
    S2DW_API_TRY
    if (!wav) return set_error(S2DWC_ERROR_ARG_INVALID, "synthesis: null wav");
    return synthesis_host(flm, wav, nullptr, scoeff, K_gamma, Phi2, Slm, J, B, N, bl_scoeff, alpha);
    S2DW_API_CATCH
}

int s2dwc_synthesis_wav2flm_dynamic(double *flm, const double *const *wav_scales, const double *scoeff,
                                    const double *K_gamma, const double *Phi2, const double *Slm, int J,
                                    int B, int N, int bl_scoeff, double alpha)
{
    S2DW_API_TRY
    if (!wav_scales) return set_error(S2DWC_ERROR_ARG_INVALID, "synthesis: null wav_scales");
    for (int j = 0; j <= J; j++)
        if (!wav_scales[j]) return set_error(S2DWC_ERROR_ARG_INVALID, "synthesis: wav_scales[%d] is null", j);
    return synthesis_host(flm, nullptr, wav_scales, scoeff, K_gamma, Phi2, Slm, J, B, N, bl_scoeff, alpha);
    S2DW_API_CATCH
}

}  // extern "C"

