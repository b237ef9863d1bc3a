// Moments of the wavelet coefficients per scale (s2dw_stat_moments,
// src/mod/s2dw_stat_mod.f90:81-275) for batches of maps resident on the GPU.
//
// Two passes over each (map, scale) block of the packed wavelet layout:
//   pass 1: sum of the (masked) coefficients and of the mask -> mean, nj;
//   pass 2: sums of s, s^2, ..., s^6 with s = w - mean over the samples whose
//           mask is 1 (all samples without a mask);
// then the reference's normalisations (n-1 variance, standardised skewness,
// excess kurtosis, fifth and excess sixth moments; zero variance -> zeros).
// Every reduction runs in a fixed order (per-block shared-memory trees, then
// the STAT_P block partials in index order), so results are bit-reproducible.
#include <cuda_runtime.h>

#include "s2dw_internal.h"

namespace s2dw {
namespace {

constexpr int STAT_T = 256;
constexpr double TOL_ZERO = 1e-12;

template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double (*sh)[STAT_T])
{
    const int t = threadIdx.x;
#pragma unroll
    for (int k = 0; k < K; k++) sh[k][t] = v[k];
    __syncthreads();
    for (int o = STAT_T / 2; o > 0; o >>= 1) {
        if (t < o) {
#pragma unroll
            for (int k = 0; k < K; k++) sh[k][t] += sh[k][t + o];
        }
        __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = sh[k][0];
}

// (map, scale) of blockIdx.y and its coefficient block
struct StatBlock {
    const double *w, *mk;
    long long n;
};
__device__ __forceinline__ StatBlock stat_block(const StatArgs &a)
{
    const int y = blockIdx.y, k = y / (a.J + 1), j = y % (a.J + 1);
    StatBlock b;
    b.w = a.wav + (size_t)k * a.wtot + a.off[j];
    b.mk = a.mask ? a.mask + a.off[j] : nullptr;
    b.n = a.off[j + 1] - a.off[j];
    return b;
}

__global__ void __launch_bounds__(STAT_T) stat_pass1(StatArgs a)
{
    __shared__ double sh[2][STAT_T];
    const StatBlock b = stat_block(a);
    double v[2] = {0.0, 0.0};
    for (long long i = (long long)blockIdx.x * STAT_T + threadIdx.x; i < b.n; i += (long long)STAT_P * STAT_T) {
        if (b.mk) {
            const double m = b.mk[i];
            if (fabs(m - 1.0) < TOL_ZERO) v[0] += b.w[i] * m;
            v[1] += m;
        } else {
            v[0] += b.w[i];
        }
    }
    block_sum<2>(v, sh);
    if (threadIdx.x == 0) {
        double *p = a.part + ((size_t)blockIdx.y * STAT_P + blockIdx.x) * 6;
        p[0] = v[0];
        p[1] = v[1];
    }
}

// mean and nj per (map, scale): the STAT_P partials in index order
__global__ void stat_mean(StatArgs a)
{
    const int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= a.nmaps * (a.J + 1)) return;
    const int j = y % (a.J + 1);
    double s = 0.0, c = 0.0;
    for (int x = 0; x < STAT_P; x++) {
        s += a.part[((size_t)y * STAT_P + x) * 6];
        c += a.part[((size_t)y * STAT_P + x) * 6 + 1];
    }
    const double nj = a.mask ? rint(c) : (double)(a.off[j + 1] - a.off[j]);
    a.mean_nj[2 * y] = s / nj;
    a.mean_nj[2 * y + 1] = nj;
}

__global__ void __launch_bounds__(STAT_T) stat_pass2(StatArgs a)
{
    __shared__ double sh[6][STAT_T];
    const StatBlock b = stat_block(a);
    const double mu = a.mean_nj[2 * blockIdx.y];
    double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (long long i = (long long)blockIdx.x * STAT_T + threadIdx.x; i < b.n; i += (long long)STAT_P * STAT_T) {
        double w = b.w[i];
        if (b.mk) {
            const double m = b.mk[i];
            if (!(fabs(m - 1.0) < TOL_ZERO)) continue;
            w *= m;
        }
        const double s = w - mu;
        double p = s * s;
        v[0] += s;
        v[1] += p;
        p *= s;
        v[2] += p;
        p *= s;
        v[3] += p;
        p *= s;
        v[4] += p;
        p *= s;
        v[5] += p;
    }
    block_sum<6>(v, sh);
    if (threadIdx.x < 6) a.part[((size_t)blockIdx.y * STAT_P + blockIdx.x) * 6 + threadIdx.x] = v[threadIdx.x];
}

// moments per (map, scale): out[y*6 + {mean, var, skew, kur, five, six}],
// flags[y] = 1 zero variance, 2 fewer than two samples
__global__ void stat_final(StatArgs a)
{
    const int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= a.nmaps * (a.J + 1)) return;
    double s[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int x = 0; x < STAT_P; x++)
#pragma unroll
        for (int k = 0; k < 6; k++) s[k] += a.part[((size_t)y * STAT_P + x) * 6 + k];
    const double mu = a.mean_nj[2 * y], nj = a.mean_nj[2 * y + 1];
    double *o = a.out + (size_t)y * 6;
    o[0] = mu;
    if (nj < 2.0) {
        a.flags[y] = 2;
        for (int k = 1; k < 6; k++) o[k] = 0.0;
        return;
    }
    const double v = (s[1] - s[0] * s[0] / nj) / (nj - 1.0);
    const double sd = sqrt(v);
    o[1] = v;
    if (v < TOL_ZERO) {
        a.flags[y] = 1;
        o[2] = o[3] = o[4] = o[5] = 0.0;
    } else {
        a.flags[y] = 0;
        o[2] = s[2] / (nj * sd * sd * sd);
        o[3] = s[3] / (nj * v * v) - 3.0;
        o[4] = s[4] / (nj * sd * sd * sd * sd * sd);
        o[5] = s[5] / (nj * v * v * v) - 15.0;
    }
}

}  // namespace

int launch_stat_moments(const StatArgs &a, cudaStream_t s)
{
    const int ny = a.nmaps * (a.J + 1);
    if (ny <= 0) return S2DWC_OK;
    dim3 grid(STAT_P, ny);
    stat_pass1<<<grid, STAT_T, 0, s>>>(a);
    stat_mean<<<(ny + 127) / 128, 128, 0, s>>>(a);
    stat_pass2<<<grid, STAT_T, 0, s>>>(a);
    stat_final<<<(ny + 127) / 128, 128, 0, s>>>(a);
    S2DW_CUDA_TRY(cudaGetLastError());
    return S2DWC_OK;
}

}  // namespace s2dw
