// Analytic FIC initialisation on the device and the Philox noise table.
//
// Analytic FIC (reference fic.cpp:130-207, called per particle on the host at
// run_CMAES.cpp:144-174 by the GPU build and inside bnm() by the CPU build):
// for every node, solve the inhibitory steady state
//     I = I0_I + wEI*S_E_ss - w_II*gamma_I*tau_I*phi_I(I)        on [0, 2]
// with Brent's method (Brent 1973, ch. 4: bracketing, inverse quadratic /
// secant steps, bisection fallback), stopping when the bracket passes the
// relative interval test |hi-lo| < 0.001*min(|lo|,|hi|) (fic.cpp:71-100:
// test_interval(lo, hi, 0, 0.001), at most 100 iterations).  Then
//     S_I = phi_I(I)*tau_I*gamma_I,
//     wIE = -(1/S_I) * (I_E_ss - I_ext - I0_E - (G*J_NMDA*SC[j,:] + wEE_j e_j) . S_E_ss).
// A failed solve or a negative wIE marks the particle unstable, and its wIE is
// then 1 on every node (run_CMAES.cpp:162-166).  One CTA per particle, one
// thread per node, FP64 throughout.
//
// Noise table: the reference draws standard normals in (ms, substep, node,
// E|I) order, one stream shared by every particle and every FIC trial
// (run_CMAES.cpp:640-657, bnm.cpp:187-188, 273-274).  The Philox mode keeps
// those semantics with a counter-based generator (noise.cuh): the value for
// (ms, substep, node, E|I) is a function of the seed and those indices only,
// so the register integrator draws it in place; the table below holds the
// same values for the kernels that read one.
#include <cstdint>
#include <cuda_runtime.h>
#include "kernels.h"
#include "noise.cuh"

namespace bnm {


template <typename R>
struct FicModel {
    __device__ static double phi_I(double II) {
        typedef Model<R> C;
        return ((C::a_I * II) - C::b_I) / (1 - exp(-1 * C::d_I * ((C::a_I * II) - C::b_I)));
    }
};

// Brent zeroin state with the documented GSL iterate/bracket interface.
struct Brent {
    double a, b, c, fa, fb, fc, d, e, lo, hi, root;
};

template <typename R>
__device__ double inh_curr(double x, double I0_I, double wEI) {
    const double S_E_ss = 0.1647572075, w_II = (double)Model<R>::w_II, gamma_I_s = 1.0, tau_I_s = 0.01;
    return I0_I + wEI * S_E_ss - w_II * gamma_I_s * tau_I_s * FicModel<R>::phi_I(x) - x;
}

template <typename R>
__device__ bool brent_step(Brent& s, double I0_I, double wEI) {
    double a = s.a, b = s.b, c = s.c, fa = s.fa, fb = s.fb, fc = s.fc, d = s.d, e = s.e;
    if ((fb > 0.0 && fc > 0.0) || (fb < 0.0 && fc < 0.0)) {
        c = a;
        fc = fa;
        d = e = b - a;
    }
    if (fabs(fc) < fabs(fb)) {
        a = b; fa = fb;
        b = c; fb = fc;
        c = a; fc = fa;
    }
    const double tol = 2.0 * 2.220446049250313e-16 * fabs(b);
    const double m = 0.5 * (c - b);
    if (fb == 0.0 || fabs(m) <= tol) {
        s.a = a; s.b = b; s.c = c; s.fa = fa; s.fb = fb; s.fc = fc; s.d = d; s.e = e;
        s.root = b;
        s.lo = (b < c) ? b : c;
        s.hi = (b < c) ? c : b;
        if (fb == 0.0) s.lo = s.hi = b;
        return true;
    }
    if (fabs(e) >= tol && fabs(fa) > fabs(fb)) {
        double p, q, r, sr = fb / fa;
        if (a == c) {
            p = 2.0 * m * sr;
            q = 1.0 - sr;
        } else {
            q = fa / fc;
            r = fb / fc;
            p = sr * (2.0 * m * q * (q - r) - (b - a) * (r - 1.0));
            q = (q - 1.0) * (r - 1.0) * (sr - 1.0);
        }
        if (p > 0.0) q = -q; else p = -p;
        const double lim1 = 3.0 * m * q - fabs(tol * q), lim2 = fabs(e * q);
        if (2.0 * p < (lim1 < lim2 ? lim1 : lim2)) {
            e = d;
            d = p / q;
        } else {
            d = m;
            e = m;
        }
    } else {
        d = m;
        e = m;
    }
    a = b;
    fa = fb;
    b += (fabs(d) > tol) ? d : (m > 0.0 ? tol : -tol);
    fb = inh_curr<R>(b, I0_I, wEI);
    if (!isfinite(fb)) return false;
    s.a = a; s.b = b; s.c = c; s.fa = fa; s.fb = fb; s.fc = fc; s.d = d; s.e = e;
    s.root = b;
    double cc = c;
    if ((fb > 0.0 && fc > 0.0) || (fb < 0.0 && fc < 0.0)) cc = a;
    s.lo = (b < cc) ? b : cc;
    s.hi = (b < cc) ? cc : b;
    return true;
}

// fic.cpp:26-55: -1 when the interval test does not pass within 100 steps.
template <typename R>
__device__ double solve_inh(double I0_I, double wEI) {
    Brent s;
    s.a = 0.0;
    s.b = 2.0;
    s.fa = inh_curr<R>(0.0, I0_I, wEI);
    s.fb = inh_curr<R>(2.0, I0_I, wEI);
    s.c = s.a;
    s.fc = s.fa;
    s.d = s.e = 2.0;
    s.root = 1.0;
    int iter = 0;
    bool ok = false;
    do {
        iter++;
        if (!brent_step<R>(s, I0_I, wEI)) break;
        const double lo = s.lo, hi = s.hi;
        const double min_abs = ((lo > 0.0 && hi > 0.0) || (lo < 0.0 && hi < 0.0)) ? fmin(fabs(lo), fabs(hi)) : 0.0;
        ok = fabs(hi - lo) < 0.001 * min_abs;
    } while (!ok && iter < 100);
    return ok ? s.root : -1.0;
}

template <typename R>
__global__ void analytic_fic_kernel(FicArgs a) {
    typedef Model<R> C;
    const int sim = blockIdx.x, N = a.N;
    __shared__ int s_bad;
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    const double I0 = (double)C::I_0;
    const double I0_E = I0 * (double)C::w_E, I0_I = I0 * (double)C::w_I;
    const double GJ = a.G[sim] * C::J_NMDA;
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        const double wEI = a.wEI[(size_t)sim * N + j], wEE = a.wEE[(size_t)sim * N + j];
        const double II = solve_inh<R>(I0_I, wEI);
        bool bad = (II == -1.0);
        double J = 1.0;
        if (!bad) {
            const double SI = FicModel<R>::phi_I(II) * 0.01 * 1.0;
            double dot = 0.0;
            const double* row = a.sc + (size_t)j * N;
            for (int k = 0; k < N; k++) {
                double kee = row[k] * GJ;
                if (k == j) kee += wEE;
                dot += kee * 0.1647572075;
            }
            J = (-1 / SI) * (0.3773805650 - (double)C::I_ext - I0_E - dot);
            bad = J < 0;
        }
        if (bad) atomicOr(&s_bad, 1);
        a.wIE[(size_t)sim * N + j] = J;
    }
    __syncthreads();
    if (s_bad)
        for (int j = threadIdx.x; j < N; j += blockDim.x) a.wIE[(size_t)sim * N + j] = 1.0;
    if (threadIdx.x == 0) a.unstable[sim] = s_bad;
}

// ------------------------------------------------------------- Philox
// The noise table in the reference's array order ([ms][substep][node][E, I],
// run_CMAES.cpp:640-657): thread i draws Philox counter i = (ms * 5 + pair) *
// N + node (philox_noise_pair) and writes that node's E and I values of the
// substeps 2 pair and 2 pair + 1.
// The table's node stride ld may exceed N (a padding node's column, left as
// it is); the values depend on N, not on ld.
__global__ void philox_fill_kernel(float* out, uint64_t n_counters, int N, int ld, uint32_t key0, uint32_t key1) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_counters;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t q = i / (uint64_t)N;  // ms * 5 + pair
        const int node = (int)(i - q * (uint64_t)N);
        const int ms = (int)(q / 5), pair = (int)(q % 5);
        const float4 v = philox_noise_pair(key0, key1, ms, pair, node, N);
        const uint64_t e0 = (((uint64_t)ms * 10 + 2 * pair) * ld + node) * 2, e1 = e0 + 2 * (uint64_t)ld;
        reinterpret_cast<float2*>(out)[e0 / 2] = make_float2(v.x, v.y);
        reinterpret_cast<float2*>(out)[e1 / 2] = make_float2(v.z, v.w);
    }
}

}  // namespace bnm

using namespace bnm;

cudaError_t bnm_launch_analytic_fic(const FicArgs& a, cudaStream_t st) {
    const int threads = a.N < 256 ? ((a.N + 31) / 32) * 32 : 256;
    if (a.fp32_consts)
        analytic_fic_kernel<float><<<a.n_sims, threads, 0, st>>>(a);
    else
        analytic_fic_kernel<double><<<a.n_sims, threads, 0, st>>>(a);
    return cudaGetLastError();
}

// n = (T + 1) * 10 * N * 2 values, i.e. (T + 1) * 5 * N Philox counters, into
// a table of node stride ld >= N.
cudaError_t bnm_launch_philox(float* out, uint64_t n, int N, int ld, uint64_t seed, int num_sms, cudaStream_t st) {
    if (N < 1 || ld < N || n % (20 * (uint64_t)N)) return cudaErrorInvalidValue;
    philox_fill_kernel<<<num_sms * 8, 256, 0, st>>>(out, n / 4, N, ld, (uint32_t)seed, (uint32_t)(seed >> 32));
    return cudaGetLastError();
}

// Known-answer support: the raw Philox4x32-10 block function of the noise
// source on the device, for n (counter[4], key[2]) inputs.
namespace bnm {
__global__ void philox_probe_kernel(const uint32_t* in6, int n, uint32_t* out4) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t c[4] = {in6[6 * i], in6[6 * i + 1], in6[6 * i + 2], in6[6 * i + 3]};
    philox4x32_10(c, in6[6 * i + 4], in6[6 * i + 5]);
    for (int k = 0; k < 4; k++) out4[4 * i + k] = c[k];
}
}  // namespace bnm

#include "../../include/bnm_b200.h"
int bnm_fail_cuda(cudaError_t e, const char* expr, const char* file, int line);

extern "C" int bnm_philox_probe(int32_t device, const uint32_t* in6, int32_t n, uint32_t* out4) {
    if (!in6 || !out4 || n < 1) return BNM_EINVAL;
    BNM_CUDA_TRY(cudaSetDevice(device));
    uint32_t *d_in = nullptr, *d_out = nullptr;
    BNM_CUDA_TRY(cudaMalloc(&d_in, (size_t)n * 6 * 4));
    cudaError_t e = cudaMalloc(&d_out, (size_t)n * 4 * 4);
    if (e == cudaSuccess) e = cudaMemcpy(d_in, in6, (size_t)n * 6 * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        bnm::philox_probe_kernel<<<(n + 127) / 128, 128>>>(d_in, n, d_out);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out4, d_out, (size_t)n * 4 * 4, cudaMemcpyDeviceToHost);
    cudaFree(d_in);
    if (d_out) cudaFree(d_out);
    BNM_CUDA_TRY(e);
    return BNM_OK;
}
