// FC, sliding-window FC, FCD, KS distance and goodness of fit on the device.
//
// Reference behaviour (CPU path, which the GPU reference approximates):
//   FC          check_fit.cpp:19-62   Pearson over kept frames, pairs i>j in
//                                    row order, optional inter-hemispheric skip
//   window FC   check_fit.cpp:79-106  windows centred ws/2 .. n-1-ws/2 by step,
//                                    [c-ws/2, c+ws/2] inclusive
//   FCD         check_fit.cpp:110-134 Pearson between window-FC vectors, i>j
//   KS          check_fit.cpp:202-210 two-sample KS of emp vs sim FCD (libks)
//   GOF         check_fit.cpp:171-215 1 - r(FC) + |dmean FC| + KS; NaN -> MAX_COST
//   FIC penalty bnm.cpp:389-405, bnm.cu:752-767
//
// B200 layout:
//   * fc_window_kernel: one CTA per (simulation, chunk of pairs).  BOLD frames
//     stream through a shared-memory ring; every pair keeps FP64 running
//     co-moments of the globally centred series, updated by one add and one
//     subtract per frame as the window slides, so window FC costs O(P) per
//     window instead of O(P*L).  Static FC comes from the same pass.  Window
//     sums over pairs (for the FCD centring) follow in window_sums_kernel,
//     FP64 in a fixed order, so the FCD does not depend on the window tile.
//   * fcd_gram_kernel: FCD = Z Z^T over the centred, unit-norm window-FC rows
//     (64x64 output tiles, FP32), lower triangle only; its epilogue drops each
//     FCD value into the KS histogram (upper_bound rank among the sorted
//     empirical FCD), so FCD never has to be sorted.
//   * gof_kernel: prefix-scan of that histogram gives the exact KS statistic;
//     FC correlation / mean difference in FP64; cost assembly.
#include <cstdint>
#include <cuda_runtime.h>
#include "kernels.h"

namespace bnm {


__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename TB, int PPT>
__global__ void __launch_bounds__(256) fc_window_kernel(FcArgs a, const TB* __restrict__ bold) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N = a.N, L = a.win_len;
    double* mean = reinterpret_cast<double*>(smem_raw);  // [N]
    double* fs = mean + N;                                // full-series sums [N]
    double* fss = fs + N;
    double* ws = fss + N;                                 // current-window sums [N]
    double* wss = ws + N;
    TB* ring = reinterpret_cast<TB*>(wss + N);            // last L frames [L][N]

    const int sim = blockIdx.x;
    const int p0 = blockIdx.y * (blockDim.x * PPT);
    const size_t base = ((size_t)sim * a.frames + a.n_vols_remove) * N;
    const int T0 = a.corr_len;

    // node means over the kept frames (FP64); the series are centred on them
    for (int n = threadIdx.x; n < N; n += blockDim.x) {
        double s = 0.0;
        for (int t = 0; t < T0; t++) s += (double)bold[base + (size_t)t * N + n];
        mean[n] = s / T0;
        fs[n] = fss[n] = ws[n] = wss[n] = 0.0;
    }
    int pi[PPT], pj[PPT];
    bool pv[PPT];
    double full[PPT], win[PPT];
#pragma unroll
    for (int u = 0; u < PPT; u++) {
        const int p = p0 + u * blockDim.x + threadIdx.x;
        pv[u] = p < a.P;
        pi[u] = pv[u] ? a.pair_i[p] : 0;
        pj[u] = pv[u] ? a.pair_j[p] : 0;
        full[u] = win[u] = 0.0;
    }
    int k = 0, lo = 0;  // current window and the first frame it covers
    bool any_nan = false;
    __syncthreads();

    auto yv = [&](int t, int n) -> double { return (double)ring[(t % L) * N + n] - mean[n]; };

    for (int t = 0; t < T0; t++) {
        for (int n = threadIdx.x; n < N; n += blockDim.x) ring[(t % L) * N + n] = bold[base + (size_t)t * N + n];
        __syncthreads();
        const bool in_win = (k < a.W) && t >= lo;
        for (int n = threadIdx.x; n < N; n += blockDim.x) {
            const double y = yv(t, n);
            fs[n] += y;
            fss[n] += y * y;
            if (in_win) {
                ws[n] += y;
                wss[n] += y * y;
            }
        }
#pragma unroll
        for (int u = 0; u < PPT; u++) {
            if (!pv[u]) continue;
            const double yy = yv(t, pi[u]) * yv(t, pj[u]);
            full[u] += yy;
            if (in_win) win[u] += yy;
        }
        if (k < a.W && t == k * a.win_step + L - 1) {
            __syncthreads();  // node window sums complete
            const double invL = 1.0 / L;
#pragma unroll
            for (int u = 0; u < PPT; u++) {
                if (!pv[u]) continue;
                const int i = pi[u], j = pj[u];
                const double cov = win[u] - ws[i] * ws[j] * invL;
                const double vi = wss[i] - ws[i] * ws[i] * invL;
                const double vj = wss[j] - ws[j] * ws[j] * invL;
                const double r = cov / sqrt(vi * vj);
                const float rf = (float)r;
                if (!(r == r) || isinf(r)) any_nan = true;
                a.wfc[((size_t)sim * a.W + k) * a.P + p0 + u * blockDim.x + threadIdx.x] = rf;
            }
            __syncthreads();  // every pair has read this window's node sums
            // slide to window k+1: drop the frames it no longer covers
            const int nlo = (k + 1) * a.win_step;
            if (nlo <= t) {
                for (int tt = lo; tt < nlo; tt++) {
                    for (int n = threadIdx.x; n < N; n += blockDim.x) {
                        const double y = yv(tt, n);
                        ws[n] -= y;
                        wss[n] -= y * y;
                    }
#pragma unroll
                    for (int u = 0; u < PPT; u++)
                        if (pv[u]) win[u] -= yv(tt, pi[u]) * yv(tt, pj[u]);
                }
            } else {
                for (int n = threadIdx.x; n < N; n += blockDim.x) ws[n] = wss[n] = 0.0;
#pragma unroll
                for (int u = 0; u < PPT; u++) win[u] = 0.0;
            }
            lo = nlo;
            k++;
        }
        __syncthreads();
    }
    // static FC over all kept frames
    const double invT = 1.0 / T0;
#pragma unroll
    for (int u = 0; u < PPT; u++) {
        if (!pv[u]) continue;
        const int i = pi[u], j = pj[u];
        const double cov = full[u] - fs[i] * fs[j] * invT;
        const double vi = fss[i] - fs[i] * fs[i] * invT;
        const double vj = fss[j] - fs[j] * fs[j] * invT;
        const double r = cov / sqrt(vi * vj);
        if (!(r == r) || isinf(r)) any_nan = true;
        a.fc[(size_t)sim * a.P + p0 + u * blockDim.x + threadIdx.x] = (float)r;
    }
    if (any_nan) atomicOr(&a.nan_flag[sim], 1);
}

// ---------------------------------------------------------------- FCD Gram

constexpr int kTile = 64, kTk = 16;

__global__ void __launch_bounds__(256) fcd_gram_kernel(FcdArgs a) {
    // blockIdx.x: lower-triangular tile index, blockIdx.y: simulation
    int t = blockIdx.x, ta = 0;
    while (t >= ta + 1) { t -= ta + 1; ta++; }
    const int tb = t;  // ta >= tb
    const int sim = blockIdx.y;
    __shared__ float As[kTk][kTile + 4];
    __shared__ float Bs[kTk][kTile + 4];
    __shared__ double mA[kTile], sA[kTile], mB[kTile], sB[kTile];
    const int a0 = ta * kTile, b0 = tb * kTile;
    const float* V = a.wfc + (size_t)sim * a.W * a.P;
    const double* ws = a.wsum + (size_t)sim * a.W * 2;
    if (threadIdx.x < kTile) {
        const int r = a0 + threadIdx.x;
        double m = 0, s = 0;
        if (r < a.W) window_norm(ws + 2 * r, a.p1 - a.p0, m, s);
        mA[threadIdx.x] = m;
        sA[threadIdx.x] = s;
    } else if (threadIdx.x < 2 * kTile) {
        const int r = b0 + threadIdx.x - kTile;
        double m = 0, s = 0;
        if (r < a.W) window_norm(ws + 2 * r, a.p1 - a.p0, m, s);
        mB[threadIdx.x - kTile] = m;
        sB[threadIdx.x - kTile] = s;
    }
    __syncthreads();
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;  // 16x16 threads, 4x4 outputs each
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.f;
    for (int k0 = a.p0; k0 < a.p1; k0 += kTk) {
        // load 64 rows x 16 columns of A and B, normalised on the fly
        for (int e = threadIdx.x; e < kTile * kTk; e += blockDim.x) {
            const int r = e / kTk, c = e % kTk;
            const int ra = a0 + r, rb = b0 + r, col = k0 + c;
            float va = 0.f, vb = 0.f;
            if (ra < a.W && col < a.p1) va = (float)(((double)V[(size_t)ra * a.P + col] - mA[r]) * sA[r]);
            if (rb < a.W && col < a.p1) vb = (float)(((double)V[(size_t)rb * a.P + col] - mB[r]) * sB[r]);
            As[c][r] = va;
            Bs[c][r] = vb;
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < kTk; c++) {
            float av[4], bv[4];
#pragma unroll
            for (int i = 0; i < 4; i++) av[i] = As[c][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; j++) bv[j] = Bs[c][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
        __syncthreads();
    }
    bool any_nan = false;
    unsigned int* hist = a.hist ? a.hist + (size_t)sim * (a.m + 1) : nullptr;
    unsigned int* eq = a.hist ? a.eq + (size_t)sim * (a.m + 1) : nullptr;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int wa = a0 + ty * 4 + i, wb = b0 + tx * 4 + j;
            if (wa < a.W && wb < wa) {
                const float v = acc[i][j];
                if (!(v == v) || isinf(v)) { any_nan = true; continue; }
                const size_t idx = (size_t)wa * (wa - 1) / 2 + wb;
                if (a.fcd) a.fcd[(size_t)sim * a.n_fcd + idx] = v;
                if (hist) {
                    int c;
                    bool equal;
                    if (a.ks_lut)
                        ks_bucket_lut(a.emp_sorted, a.ks_lut, a.m, (double)v, c, equal);
                    else
                        ks_bucket(a.emp_sorted, a.m, (double)v, c, equal);
                    atomicAdd(&hist[c], 1u);
                    if (equal) atomicAdd(&eq[c], 1u);
                }
            }
        }
    if (any_nan && a.nan_flag) atomicOr(&a.nan_flag[sim], 1);
}

// ------------------------------------------------------------ KS + GOF

__device__ double block_sum(double v, double* sh) {
    v = warp_sum(v);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += sh[w];
    return s;
}

__device__ double block_max(double v, double* sh) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s = fmax(s, sh[w]);
    return s;
}

__global__ void __launch_bounds__(1024) gof_kernel(GofArgs a) {
    __shared__ double sh[32];
    __shared__ unsigned long long seg[1024];
    const int sim = blockIdx.x;
    // FC: Pearson with the empirical FC, and mean difference (FP64, two passes)
    const float* fc = a.fc + (size_t)sim * a.P;
    double s = 0.0;
    for (int p = threadIdx.x; p < a.P; p += blockDim.x) s += fc[p];
    const double msim = block_sum(s, sh) / a.P;
    double sxy = 0, sxx = 0, syy = 0;
    for (int p = threadIdx.x; p < a.P; p += blockDim.x) {
        const double dx = a.emp_fc[p] - a.emp_fc_mean, dy = (double)fc[p] - msim;
        sxy += dx * dy;
        sxx += dx * dx;
        syy += dy * dy;
    }
    sxy = block_sum(sxy, sh);
    sxx = block_sum(sxx, sh);
    syy = block_sum(syy, sh);
    const double r = sxy / (sqrt(sxx) * sqrt(syy));
    // KS: D = max over jump points c of |c/m - F_sim| just before/at the point
    double D = 0.0;
    if (!a.no_fcd) {
        const int nb = a.m + 1;
        const unsigned int* h = a.hist + (size_t)sim * nb;
        const unsigned int* q = a.eq + (size_t)sim * nb;
        const int per = (nb + blockDim.x - 1) / blockDim.x;
        const int c0 = threadIdx.x * per, c1 = min(nb, c0 + per);
        unsigned long long loc = 0;
        for (int c = c0; c < c1; c++) loc += h[c];
        seg[threadIdx.x] = loc;
        __syncthreads();
        if (threadIdx.x == 0) {  // exclusive scan of segment totals
            unsigned long long run = 0;
            for (int w = 0; w < (int)blockDim.x; w++) {
                const unsigned long long v = seg[w];
                seg[w] = run;
                run += v;
            }
        }
        __syncthreads();
        unsigned long long H = seg[threadIdx.x];  // sims with rank < c0
        const double invm = 1.0 / a.m, invn = 1.0 / a.n_fcd;
        double dmax = 0.0;
        for (int c = c0; c < c1; c++) {
            const double Fe = c * invm;
            if (a.valid[c]) {
                dmax = fmax(dmax, fabs(Fe - (double)(H + q[c]) * invn));
                dmax = fmax(dmax, fabs(Fe - (double)(H + h[c]) * invn));
            }
            H += h[c];
        }
        D = block_max(dmax, sh);
    }
    double pen = 0.0;
    if (a.calc_fic_penalty) {
        double ps = 0.0;
        for (int j = threadIdx.x; j < a.N; j += blockDim.x) {
            const double d = fabs(a.ext[((size_t)sim * 6 + 2) * a.N + j] - 3);
            if (d > 1) ps += 1 - exp(-0.05 * (d - 1));
        }
        pen = block_sum(ps, sh) * a.fic_penalty_scale / a.N;
        if (a.fic_reject_failed && a.failed[sim]) pen += 1;
    }
    if (threadIdx.x == 0) {
        const double diff = fabs(a.emp_fc_mean - msim);
        double c = 1 - r + (a.use_fc_diff ? diff : 0.0) + D;
        const bool bad = a.nan_flag[sim] != 0 || !(r == r);
        if (bad) c = a.max_cost;
        a.cost[sim] = c;
        a.fc_corr[sim] = r;
        a.fc_diff[sim] = diff;
        a.fcd_ks[sim] = D;
        a.fic_penalty[sim] = a.calc_fic_penalty ? pen : 0.0;
    }
}

}  // namespace bnm

using namespace bnm;

template <typename TB, int PPT>
static cudaError_t launch_fc_window_t(const FcArgs& a, const TB* bold, cudaStream_t st) {
    constexpr int TPB = 256;
    const int chunks = (a.P + TPB * PPT - 1) / (TPB * PPT);
    const size_t smem = (size_t)a.N * 5 * sizeof(double) + (size_t)a.win_len * a.N * sizeof(TB);
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(fc_window_kernel<TB, PPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid(a.n_sims, chunks);
    fc_window_kernel<TB, PPT><<<grid, TPB, smem, st>>>(a, bold);
    return cudaGetLastError();
}

// The window tile: each CTA of 256 threads carries 256 ppt pairs through the
// frames (ppt in {1, 2, 4, 8}); fewer pairs per CTA give more CTAs but repeat
// the node means and the frame ring per CTA.  The plan's tuner picks ppt.
template <typename TB>
static cudaError_t launch_fc_window(const FcArgs& a, const TB* bold, cudaStream_t st) {
    switch (a.ppt ? a.ppt : 4) {
        case 1: return launch_fc_window_t<TB, 1>(a, bold, st);
        case 2: return launch_fc_window_t<TB, 2>(a, bold, st);
        case 4: return launch_fc_window_t<TB, 4>(a, bold, st);
        case 8: return launch_fc_window_t<TB, 8>(a, bold, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t bnm_launch_fc_window(const FcArgs& a, cudaStream_t st) {
    cudaError_t e = a.bold_f64 ? launch_fc_window<double>(a, a.bold_f64, st) : launch_fc_window<float>(a, a.bold, st);
    if (e != cudaSuccess || a.W < 1) return e;
    // The window rows' sums over all pairs, in a fixed order: the same BOLD
    // gives the same FCD whatever the window tile and the launch order.
    return bnm_launch_window_sums(a.wfc, a.n_sims, a.W, a.P, 0, a.P, a.wsum, st);
}

// Window-FC sums over a pair range, one CTA per (window, simulation): the
// centring of the hemisphere FCDs (window_fc_stats with save_hemis,
// bnm.cu:436-496).
__global__ void __launch_bounds__(256) window_sums_kernel(const float* wfc, int W, int P, int p0, int p1,
                                                          double* out) {
    __shared__ double sh[16];
    const int w = blockIdx.x, sim = blockIdx.y;
    const float* v = wfc + ((size_t)sim * W + w) * P;
    double s = 0.0, ss = 0.0;
    for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
        const double x = v[p];
        s += x;
        ss += x * x;
    }
    s = warp_sum(s);
    ss = warp_sum(ss);
    if ((threadIdx.x & 31) == 0) {
        sh[threadIdx.x >> 5] = s;
        sh[8 + (threadIdx.x >> 5)] = ss;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) {
            a += sh[k];
            b += sh[8 + k];
        }
        out[((size_t)sim * W + w) * 2] = a;
        out[((size_t)sim * W + w) * 2 + 1] = b;
    }
}

cudaError_t bnm_launch_window_sums(const float* wfc, int n_sims, int W, int P, int p0, int p1, double* wsum_out,
                                   cudaStream_t st) {
    if (p0 < 0 || p1 > P || p1 - p0 < 2) return cudaErrorInvalidValue;
    window_sums_kernel<<<dim3(W, n_sims), 256, 0, st>>>(wfc, W, P, p0, p1, wsum_out);
    return cudaGetLastError();
}

cudaError_t bnm_launch_fcd(FcdArgs a, cudaStream_t st) {
    a.tiles = (a.W + kTile - 1) / kTile;
    dim3 grid(a.tiles * (a.tiles + 1) / 2, a.n_sims);
    fcd_gram_kernel<<<grid, 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t bnm_launch_gof(const GofArgs& a, cudaStream_t st) {
    gof_kernel<<<a.n_sims, 1024, 0, st>>>(a);
    return cudaGetLastError();
}
