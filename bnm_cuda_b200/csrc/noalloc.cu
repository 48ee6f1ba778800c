// Goodness of fit of BOLD series that are already on the device, using no
// allocated memory: bnm_gof_noalloc.
//
// Who needs it: hosts that keep the device allocator for themselves -- an
// embedding framework with its own caching allocator or a fixed memory
// budget, a real-time or streaming loop that must not call cudaMalloc /
// cudaFree (cudaFree synchronises the whole device, stalling every other
// stream), or a caller that has already carved its device memory and can
// only hand over input and output buffers.  They get the same FC, window-FC,
// FCD, KS and cost kernels as a plan, with every intermediate placed in one
// file-scope device array instead of plan-owned buffers.
//
// Limits and sharing rules:
//   * the scratch array is BNM_NOALLOC_SCRATCH_BYTES (32 MiB) per device and
//     stays resident on every GPU that loads the library until the process
//     exits;  a call whose intermediates do not fit is rejected (BNM_EINVAL)
//     before any device work;
//   * every call uses the same array and leaves its contents behind; the call
//     clears what must start at zero itself, but two calls that overlap on the
//     GPU (different streams or threads without ordering) race on it;
//   * the first call on a device looks up the array's device address (a
//     one-time set-up per device); make that first call before any stream
//     capture.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/bnm_b200.h"
#include "kernels.h"

int bnm_fail_cuda(cudaError_t e, const char* expr, const char* file, int line);
int bnm_fail_msg(int code, const char* msg);

namespace {

constexpr size_t kScratchBytes = BNM_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of g_noalloc_scratch per device (host code may not use the
// symbol itself as a pointer).
constexpr int kMaxDevices = 64;
unsigned char* g_scratch_ptr[kMaxDevices] = {};
std::mutex g_scratch_mu;

int scratch_for(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices) return bnm_fail_msg(BNM_EINVAL, "device index out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return bnm_fail_cuda(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
        g_scratch_ptr[device] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_ptr[device];
    return BNM_OK;
}

// Lower-triangle pair table of run_CMAES.cpp:505-524 (i > j, i outer, j
// inner; with exc_interhem the pairs that cross the N/2 split are skipped):
// one thread per row i writes its pairs at the row's closed-form offset.
__global__ void pair_table_kernel(int N, int exc, int* pi, int* pj) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int h = N / 2;
    long long start;
    int j0;
    if (!exc) {
        start = (long long)i * (i - 1) / 2;
        j0 = 0;
    } else if (i < h) {
        start = (long long)i * (i - 1) / 2;
        j0 = 0;
    } else {
        start = (long long)h * (h - 1) / 2 + (long long)(i - h) * (i - h - 1) / 2;
        j0 = h;
    }
    for (int j = j0; j < i; j++) {
        pi[start + (j - j0)] = i;
        pj[start + (j - j0)] = j;
    }
}

// KS jump flags of the sorted empirical FCD: rank c (0..m) is a point where
// F_emp jumps (c == 0, c == m, or e[c-1] < e[c]).
__global__ void ks_valid_kernel(const double* e, int m, unsigned char* valid) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c <= m; c += gridDim.x * blockDim.x)
        valid[c] = (c == 0 || c == m) ? 1 : (e[c - 1] < e[c] ? 1 : 0);
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

extern "C" int bnm_gof_noalloc(const float* d_bold, int32_t n, int32_t frames, int32_t nodes, int32_t n_vols_remove,
                               int32_t window_size, int32_t window_step, int32_t exc_interhem, int32_t use_fc_diff,
                               double max_cost, const double* emp_fc, int32_t n_emp_fc, const double* emp_fcd_sorted,
                               int32_t n_emp_fcd, double* d_out, void* stream) {
    using namespace bnm;
    if (!d_bold || !d_out || !emp_fc || !emp_fcd_sorted) return bnm_fail_msg(BNM_EINVAL, "null argument");
    const int N = nodes;
    if (n < 1 || N < 2 || frames < 2 || window_step < 1 || window_size < 0 || n_vols_remove < 0)
        return bnm_fail_msg(BNM_EINVAL, "bad sizes");
    if (exc_interhem && (N % 2)) return bnm_fail_msg(BNM_EINVAL, "exc_interhem needs an even node count");
    const int corr_len = frames - n_vols_remove;
    if (corr_len < 2) return bnm_fail_msg(BNM_EINVAL, "fewer than 2 frames after removal");
    const int P = N * (N - 1) / 2 - (exc_interhem ? (N / 2) * (N / 2) : 0);
    if (P < 2) return bnm_fail_msg(BNM_EINVAL, "fewer than 2 node pairs (FC correlation undefined)");
    if (n_emp_fc != P) return bnm_fail_msg(BNM_EINVAL, "empirical FC length does not match the pair count");
    const int h = window_size / 2, L = 2 * h + 1, first = h, last = corr_len - 1 - h;
    const int W = last >= first ? (last - first) / window_step + 1 : 0;
    if (W < 2) return bnm_fail_msg(BNM_EINVAL, "need at least 2 FCD windows");
    const int m = n_emp_fcd;
    if (m < 1) return bnm_fail_msg(BNM_EINVAL, "empirical FCD is empty");
    for (int c = 1; c < m; c++)
        if (!(emp_fcd_sorted[c - 1] <= emp_fcd_sorted[c]))
            return bnm_fail_msg(BNM_EINVAL, "empirical FCD must be sorted ascending");
    double mfc = 0.0;
    for (int p = 0; p < P; p++) mfc += emp_fc[p];
    mfc /= P;

    // scratch layout (256-byte aligned pieces)
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t at = off;
        off = align256(off + bytes);
        return at;
    };
    const size_t o_pi = take((size_t)P * 4), o_pj = take((size_t)P * 4);
    const size_t o_efc = take((size_t)P * 8), o_es = take((size_t)m * 8), o_valid = take((size_t)m + 1);
    const size_t o_fc = take((size_t)n * P * 4), o_wfc = take((size_t)n * W * P * 4);
    const size_t o_wsum = take((size_t)n * W * 2 * 8), o_hist = take((size_t)n * (m + 1) * 4);
    const size_t o_eq = take((size_t)n * (m + 1) * 4), o_nan = take((size_t)n * 4), o_zero = take(8 * (size_t)n + 8);
    const size_t needed = off;
    if (needed > kScratchBytes) {
        char msg[256];
        std::snprintf(msg, sizeof msg,
                      "needs %zu bytes of scratch; the static scratch holds %zu (BNM_NOALLOC_SCRATCH_BYTES): "
                      "pass fewer series per call",
                      needed, kScratchBytes);
        return bnm_fail_msg(BNM_EINVAL, msg);
    }
    int device = 0;
    BNM_CUDA_TRY(cudaGetDevice(&device));
    unsigned char* s = nullptr;
    int rc = scratch_for(device, &s);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    int* pi = reinterpret_cast<int*>(s + o_pi);
    int* pj = reinterpret_cast<int*>(s + o_pj);
    double* efc = reinterpret_cast<double*>(s + o_efc);
    double* es = reinterpret_cast<double*>(s + o_es);
    unsigned char* valid = s + o_valid;
    // inputs copied into scratch; accumulators cleared (the array keeps the
    // previous call's contents)
    BNM_CUDA_TRY(cudaMemcpyAsync(efc, emp_fc, (size_t)P * 8, cudaMemcpyHostToDevice, st));
    BNM_CUDA_TRY(cudaMemcpyAsync(es, emp_fcd_sorted, (size_t)m * 8, cudaMemcpyHostToDevice, st));
    BNM_CUDA_TRY(cudaMemsetAsync(s + o_wsum, 0, (size_t)n * W * 2 * 8, st));
    BNM_CUDA_TRY(cudaMemsetAsync(s + o_hist, 0, (size_t)n * (m + 1) * 4, st));
    BNM_CUDA_TRY(cudaMemsetAsync(s + o_eq, 0, (size_t)n * (m + 1) * 4, st));
    BNM_CUDA_TRY(cudaMemsetAsync(s + o_nan, 0, (size_t)n * 4, st));
    BNM_CUDA_TRY(cudaMemsetAsync(s + o_zero, 0, 8 * (size_t)n + 8, st));
    pair_table_kernel<<<(N + 127) / 128, 128, 0, st>>>(N, exc_interhem, pi, pj);
    ks_valid_kernel<<<(m + 256) / 256 < 1024 ? (m + 256) / 256 : 1024, 256, 0, st>>>(es, m, valid);
    BNM_CUDA_TRY(cudaGetLastError());

    FcArgs fa;
    std::memset(&fa, 0, sizeof fa);
    fa.N = N;
    fa.n_sims = n;
    fa.frames = frames;
    fa.n_vols_remove = n_vols_remove;
    fa.corr_len = corr_len;
    fa.P = P;
    fa.pair_i = pi;
    fa.pair_j = pj;
    fa.W = W;
    fa.win_len = L;
    fa.win_step = window_step;
    fa.bold = d_bold;
    fa.bold_f64 = nullptr;
    fa.fc = reinterpret_cast<float*>(s + o_fc);
    fa.wfc = reinterpret_cast<float*>(s + o_wfc);
    fa.wsum = reinterpret_cast<double*>(s + o_wsum);
    fa.nan_flag = reinterpret_cast<int*>(s + o_nan);
    BNM_CUDA_TRY(bnm_launch_fc_window(fa, st));

    FcdArgs da;
    std::memset(&da, 0, sizeof da);  // no bucket table: plain rank search
    da.n_sims = n;
    da.W = W;
    da.P = P;
    da.wfc = fa.wfc;
    da.wsum = fa.wsum;
    da.fcd = nullptr;
    da.n_fcd = W * (W - 1) / 2;
    da.emp_sorted = es;
    da.m = m;
    da.hist = reinterpret_cast<unsigned int*>(s + o_hist);
    da.eq = reinterpret_cast<unsigned int*>(s + o_eq);
    da.nan_flag = fa.nan_flag;
    da.p0 = 0;
    da.p1 = P;
    BNM_CUDA_TRY(bnm_launch_fcd(da, st));

    GofArgs ga;
    std::memset(&ga, 0, sizeof ga);
    ga.n_sims = n;
    ga.N = N;
    ga.P = P;
    ga.n_fcd = da.n_fcd;
    ga.m = m;
    ga.fc = fa.fc;
    ga.emp_fc = efc;
    ga.emp_fc_mean = mfc;
    ga.hist = da.hist;
    ga.eq = da.eq;
    ga.valid = valid;
    ga.ext = reinterpret_cast<const double*>(s + o_zero);
    ga.failed = reinterpret_cast<const int*>(s + o_zero);
    ga.nan_flag = fa.nan_flag;
    ga.use_fc_diff = use_fc_diff;
    ga.calc_fic_penalty = 0;
    ga.fic_reject_failed = 0;
    ga.no_fcd = 0;
    ga.max_cost = max_cost;
    ga.fic_penalty_scale = 0.0;
    // d_out rows: cost, fc_corr, fc_diff, fcd_ks, (fic penalty slot, 0)
    ga.cost = d_out;
    ga.fc_corr = d_out + n;
    ga.fc_diff = d_out + 2 * (size_t)n;
    ga.fcd_ks = d_out + 3 * (size_t)n;
    ga.fic_penalty = d_out + 4 * (size_t)n;
    BNM_CUDA_TRY(bnm_launch_gof(ga, st));
    return BNM_OK;
}
