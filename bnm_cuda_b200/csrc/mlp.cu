// MLP surrogate of the simulate-and-fit cost (no counterpart in the
// reference): maps (G, wEE, wEI, SC spectral summary) to the fit terms so that
// oversampled CMA-ES candidates can be pre-screened before simulation.
//
// Network: in -> [hidden, ReLU] x layers -> out, weights kept in FP32 (master
// copy for Adam) and rounded to BF16 for the forward GEMMs; activations are
// stored in BF16; every GEMM accumulates in FP32.  Training (MSE loss, Adam)
// runs entirely on the device with this file's kernels:
//   gemm_bf16_kernel  C = A B (+bias, ReLU) on mma.sync m16n8k16 BF16 tensor
//                     cores with FP32 accumulation; operands are read through
//                     strides (so W, W^T and X^T need no copies) and A may be
//                     multiplied by a ReLU mask (the backward of the ReLU fused
//                     into the dX and dW GEMMs);
//   bias_grad_kernel, mse_grad_kernel, adam_kernel, cast kernels.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

#include <cuda_bf16.h>

#include "../../include/bnm_b200.h"
#include "kernels.h"

int bnm_fail_cuda(cudaError_t e, const char* expr, const char* file, int line);
int bnm_fail_msg(int code, const char* msg);

namespace {

constexpr int TM = 64, TN = 64, TK = 32, SPAD = 8;  // CTA tile and shared-memory row padding

struct GemmOp {
    int M, N, K;
    const void* A;       // A(m,k) = A[m*sam + k*sak]
    long long sam, sak;
    int a_f32;           // A element type: 1 = float, 0 = bf16
    const __nv_bfloat16* mask;  // optional: A(m,k) *= (mask[m*smm + k*smk] > 0)
    long long smm, smk;
    const void* B;       // B(k,n) = B[k*sbk + n*sbn]
    long long sbk, sbn;
    int b_f32;
    const float* bias;   // optional, [N]
    int relu;            // epilogue ReLU
    void* C;             // C[m*ldc + n]
    long long ldc;
    int c_f32;           // 1: float output, 0: bf16 output
    float alpha;
};

__device__ __forceinline__ float load_elem(const void* p, long long i, int f32) {
    return f32 ? static_cast<const float*>(p)[i] : __bfloat162float(static_cast<const __nv_bfloat16*>(p)[i]);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// 4 warps, each a 32x32 piece of the 64x64 CTA tile: 2 (m16) x 4 (n8) mma tiles.
__global__ void __launch_bounds__(128) gemm_bf16_kernel(GemmOp op) {
    __shared__ __align__(16) __nv_bfloat16 As[TM][TK + SPAD];  // [m][k]
    __shared__ __align__(16) __nv_bfloat16 Bs[TN][TK + SPAD];  // [n][k]
    const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int g = lane >> 2, t = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int jn = 0; jn < 4; jn++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[i][jn][q] = 0.f;

    for (int k0 = 0; k0 < op.K; k0 += TK) {
        for (int e = threadIdx.x; e < TM * TK; e += blockDim.x) {
            const int r = e / TK, c = e % TK, m = m0 + r, k = k0 + c;
            float va = 0.f;
            if (m < op.M && k < op.K) {
                va = load_elem(op.A, m * op.sam + k * op.sak, op.a_f32);
                if (op.mask && !(__bfloat162float(op.mask[m * op.smm + k * op.smk]) > 0.f)) va = 0.f;
            }
            As[r][c] = __float2bfloat16_rn(va);
        }
        for (int e = threadIdx.x; e < TN * TK; e += blockDim.x) {
            const int r = e / TK, c = e % TK, n = n0 + r, k = k0 + c;
            const float vb = (n < op.N && k < op.K) ? load_elem(op.B, k * op.sbk + n * op.sbn, op.b_f32) : 0.f;
            Bs[r][c] = __float2bfloat16_rn(vb);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TK; kk += 16) {
            uint32_t af[2][4], bf[4][2];
#pragma unroll
            for (int i = 0; i < 2; i++) {
                const int r = wm + i * 16 + g;
                af[i][0] = *reinterpret_cast<const uint32_t*>(&As[r][kk + 2 * t]);
                af[i][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + 2 * t]);
                af[i][2] = *reinterpret_cast<const uint32_t*>(&As[r][kk + 2 * t + 8]);
                af[i][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + 2 * t + 8]);
            }
#pragma unroll
            for (int jn = 0; jn < 4; jn++) {
                const int c = wn + jn * 8 + g;
                bf[jn][0] = *reinterpret_cast<const uint32_t*>(&Bs[c][kk + 2 * t]);
                bf[jn][1] = *reinterpret_cast<const uint32_t*>(&Bs[c][kk + 2 * t + 8]);
            }
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int jn = 0; jn < 4; jn++) mma_bf16(acc[i][jn], af[i], bf[jn]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int jn = 0; jn < 4; jn++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int m = m0 + wm + i * 16 + g + (q >= 2 ? 8 : 0);
                const int n = n0 + wn + jn * 8 + 2 * t + (q & 1);
                if (m >= op.M || n >= op.N) continue;
                float v = op.alpha * acc[i][jn][q];
                if (op.bias) v += op.bias[n];
                if (op.relu) v = fmaxf(v, 0.f);
                if (op.c_f32)
                    static_cast<float*>(op.C)[m * op.ldc + n] = v;
                else
                    static_cast<__nv_bfloat16*>(op.C)[m * op.ldc + n] = __float2bfloat16_rn(v);
            }
}

// db[o] = sum_b dY[b][o] * (mask? Y[b][o] > 0)
__global__ void bias_grad_kernel(const float* dY, const __nv_bfloat16* mask, int B, int O, float* db) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= O) return;
    float s = 0.f;
    for (int b = 0; b < B; b++) {
        const float d = dY[(size_t)b * O + o];
        if (!mask || __bfloat162float(mask[(size_t)b * O + o]) > 0.f) s += d;
    }
    db[o] = s;
}

// MSE over the batch: loss = mean_b sum_o (y - t)^2 / O; dY = 2 (y - t) / (B O)
__global__ void mse_grad_kernel(const float* Y, const float* T, int B, int O, float* dY, float* loss) {
    __shared__ float red[256];
    float s = 0.f;
    for (int i = threadIdx.x; i < B * O; i += blockDim.x) {
        const float d = Y[i] - T[i];
        dY[i] = 2.f * d / (float)(B * O);
        s += d * d;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss = red[0] / (float)(B * O);
}

__global__ void adam_kernel(float* w, const float* g, float* m, float* v, __nv_bfloat16* w16, long long n, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (w16) w16[i] = __float2bfloat16_rn(wi);
    }
}

__global__ void to_bf16_kernel(const float* x, __nv_bfloat16* y, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16_rn(x[i]);
}

__global__ void gather_rows_kernel(const float* X, const int* idx, int n, int d, float* out) {
    const long long total = (long long)n * d;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const long long r = e / d, c = e % d;
        out[e] = X[(long long)idx[r] * d + c];
    }
}

cudaError_t gemm(const GemmOp& op, cudaStream_t st) {
    dim3 grid((op.N + TN - 1) / TN, (op.M + TM - 1) / TM);
    gemm_bf16_kernel<<<grid, 128, 0, st>>>(op);
    return cudaGetLastError();
}

GemmOp base_op() {
    GemmOp o;
    std::memset(&o, 0, sizeof o);
    o.alpha = 1.f;
    return o;
}

}  // namespace

struct bnm_mlp {
    int in = 0, hidden = 0, layers = 0, out = 0, max_batch = 0, device = 0;
    int L = 0;  // number of linear layers = layers + 1
    std::vector<int> din, dout;
    std::vector<long long> woff, boff;  // offsets into the flat parameter vector
    long long n_params = 0;
    cudaStream_t st = nullptr;
    float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;  // flat [W_l (out x in), b_l (out)]...
    __nv_bfloat16* w16 = nullptr;
    std::vector<__nv_bfloat16*> act;  // act[0] = input (bf16), act[l] = hidden outputs (bf16)
    float* yout = nullptr;            // [max_batch][out] last-layer output (f32)
    float *dA = nullptr, *dB = nullptr;  // gradient ping-pong [max_batch][max width]
    float* loss = nullptr;
    float *xin = nullptr, *tgt = nullptr;  // staged batch input / target (f32)
    float *data_x = nullptr, *data_y = nullptr;  // training set on the device
    int* idx = nullptr;
    long long data_n = 0;
    int adam_t = 0;
    std::vector<void*> allocs;
};

static int mlp_alloc(bnm_mlp* p, void** ptr, size_t bytes) {
    cudaError_t e = cudaMalloc(ptr, bytes ? bytes : 16);
    if (e != cudaSuccess) return bnm_fail_cuda(e, "cudaMalloc", __FILE__, __LINE__);
    p->allocs.push_back(*ptr);
    return BNM_OK;
}

extern "C" void bnm_mlp_destroy(bnm_mlp* p) {
    if (!p) return;
    cudaSetDevice(p->device);
    if (p->st) cudaStreamSynchronize(p->st);
    for (void* a : p->allocs) cudaFree(a);
    if (p->st) cudaStreamDestroy(p->st);
    delete p;
}

extern "C" int bnm_mlp_create(int32_t in_dim, int32_t hidden, int32_t layers, int32_t out_dim, int32_t max_batch,
                              uint64_t seed, int32_t device, bnm_mlp** out) {
    if (!out || in_dim < 1 || hidden < 1 || layers < 1 || out_dim < 1 || max_batch < 1)
        return bnm_fail_msg(BNM_EINVAL, "bad MLP sizes");
    *out = nullptr;
    bnm_mlp* p = new bnm_mlp();
    p->in = in_dim;
    p->hidden = hidden;
    p->layers = layers;
    p->out = out_dim;
    p->max_batch = max_batch;
    p->device = device;
    p->L = layers + 1;
    for (int l = 0; l < p->L; l++) {
        p->din.push_back(l == 0 ? in_dim : hidden);
        p->dout.push_back(l == p->L - 1 ? out_dim : hidden);
        p->woff.push_back(p->n_params);
        p->n_params += (long long)p->din[l] * p->dout[l];
        p->boff.push_back(p->n_params);
        p->n_params += p->dout[l];
    }
    int rc = BNM_OK;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        rc = bnm_fail_cuda(e, "cudaSetDevice/cudaStreamCreate", __FILE__, __LINE__);
        bnm_mlp_destroy(p);
        return rc;
    }
    const size_t np = (size_t)p->n_params;
    const int wmax = std::max(std::max(in_dim, hidden), out_dim);
    void* ptr;
#define MLP_ALLOC(field, bytes)                                   \
    if ((rc = mlp_alloc(p, &ptr, (bytes)))) {                     \
        bnm_mlp_destroy(p);                                       \
        return rc;                                                \
    }                                                             \
    p->field = static_cast<decltype(p->field)>(ptr);
    MLP_ALLOC(w, np * 4);
    MLP_ALLOC(g, np * 4);
    MLP_ALLOC(m, np * 4);
    MLP_ALLOC(v, np * 4);
    MLP_ALLOC(w16, np * 2);
    MLP_ALLOC(yout, (size_t)max_batch * out_dim * 4);
    MLP_ALLOC(dA, (size_t)max_batch * wmax * 4);
    MLP_ALLOC(dB, (size_t)max_batch * wmax * 4);
    MLP_ALLOC(loss, 16);
    MLP_ALLOC(xin, (size_t)max_batch * in_dim * 4);
    MLP_ALLOC(tgt, (size_t)max_batch * out_dim * 4);
    MLP_ALLOC(idx, (size_t)max_batch * 4);
#undef MLP_ALLOC
    p->act.assign(p->L, nullptr);
    for (int l = 0; l < p->L; l++) {
        if ((rc = mlp_alloc(p, &ptr, (size_t)max_batch * p->din[l] * 2))) {
            bnm_mlp_destroy(p);
            return rc;
        }
        p->act[l] = static_cast<__nv_bfloat16*>(ptr);
    }
    // He-uniform initialisation (host, seeded), zero biases; Adam state zero
    std::vector<float> w0(np, 0.f);
    std::mt19937_64 gen(seed);
    for (int l = 0; l < p->L; l++) {
        const float lim = std::sqrt(6.0f / (float)p->din[l]);
        std::uniform_real_distribution<float> U(-lim, lim);
        for (long long i = 0; i < (long long)p->din[l] * p->dout[l]; i++) w0[p->woff[l] + i] = U(gen);
    }
    e = cudaMemcpy(p->w, w0.data(), np * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(p->m, 0, np * 4);
    if (e == cudaSuccess) e = cudaMemset(p->v, 0, np * 4);
    if (e == cudaSuccess) {
        to_bf16_kernel<<<256, 256, 0, p->st>>>(p->w, p->w16, (long long)np);
        e = cudaStreamSynchronize(p->st);
    }
    if (e != cudaSuccess) {
        rc = bnm_fail_cuda(e, "MLP initialisation", __FILE__, __LINE__);
        bnm_mlp_destroy(p);
        return rc;
    }
    *out = p;
    return BNM_OK;
}

// forward pass of a staged batch (xin f32 [B][in]) into yout
static int forward(bnm_mlp* p, int B) {
    to_bf16_kernel<<<64, 256, 0, p->st>>>(p->xin, p->act[0], (long long)B * p->in);
    for (int l = 0; l < p->L; l++) {
        GemmOp o = base_op();
        o.M = B;
        o.N = p->dout[l];
        o.K = p->din[l];
        o.A = p->act[l];
        o.sam = p->din[l];
        o.sak = 1;
        o.B = p->w16 + p->woff[l];  // W_l [out][in]: B(k=in, n=out) = W[n*in + k]
        o.sbk = 1;
        o.sbn = p->din[l];
        o.bias = p->w + p->boff[l];
        const bool last = l == p->L - 1;
        o.relu = !last;
        o.C = last ? (void*)p->yout : (void*)p->act[l + 1];
        o.ldc = p->dout[l];
        o.c_f32 = last;
        BNM_CUDA_TRY(gemm(o, p->st));
    }
    return BNM_OK;
}

// loss and gradients of the staged batch (xin, tgt) into p->g
static int backward(bnm_mlp* p, int B) {
    mse_grad_kernel<<<1, 256, 0, p->st>>>(p->yout, p->tgt, B, p->out, p->dA, p->loss);
    float* dY = p->dA;
    float* dX = p->dB;
    for (int l = p->L - 1; l >= 0; l--) {
        const bool last = l == p->L - 1;
        // the ReLU of layer l's output (hidden layers) masks dY
        const __nv_bfloat16* mask = last ? nullptr : p->act[l + 1];
        bias_grad_kernel<<<(p->dout[l] + 127) / 128, 128, 0, p->st>>>(dY, mask, B, p->dout[l], p->g + p->boff[l]);
        // dW[o][i] = sum_b dZ[b][o] X[b][i]
        GemmOp gw = base_op();
        gw.M = p->dout[l];
        gw.N = p->din[l];
        gw.K = B;
        gw.A = dY;
        gw.a_f32 = 1;
        gw.sam = 1;
        gw.sak = p->dout[l];
        gw.mask = mask;
        gw.smm = 1;
        gw.smk = p->dout[l];
        gw.B = p->act[l];
        gw.sbk = p->din[l];
        gw.sbn = 1;
        gw.C = p->g + p->woff[l];
        gw.ldc = p->din[l];
        gw.c_f32 = 1;
        BNM_CUDA_TRY(gemm(gw, p->st));
        if (l == 0) break;
        // dX[b][i] = sum_o dZ[b][o] W[o][i]
        GemmOp gx = base_op();
        gx.M = B;
        gx.N = p->din[l];
        gx.K = p->dout[l];
        gx.A = dY;
        gx.a_f32 = 1;
        gx.sam = p->dout[l];
        gx.sak = 1;
        gx.mask = mask;
        gx.smm = p->dout[l];
        gx.smk = 1;
        gx.B = p->w16 + p->woff[l];
        gx.sbk = p->din[l];
        gx.sbn = 1;
        gx.C = dX;
        gx.ldc = p->din[l];
        gx.c_f32 = 1;
        BNM_CUDA_TRY(gemm(gx, p->st));
        std::swap(dY, dX);
    }
    return BNM_OK;
}

extern "C" int bnm_mlp_predict(bnm_mlp* p, const float* X, int32_t n, float* Y) {
    if (!p || !X || !Y || n < 0) return bnm_fail_msg(BNM_EINVAL, "bad predict arguments");
    BNM_CUDA_TRY(cudaSetDevice(p->device));
    for (int s = 0; s < n; s += p->max_batch) {
        const int B = std::min(p->max_batch, n - s);
        BNM_CUDA_TRY(cudaMemcpyAsync(p->xin, X + (size_t)s * p->in, (size_t)B * p->in * 4, cudaMemcpyHostToDevice, p->st));
        int rc = forward(p, B);
        if (rc) return rc;
        BNM_CUDA_TRY(cudaMemcpyAsync(Y + (size_t)s * p->out, p->yout, (size_t)B * p->out * 4, cudaMemcpyDeviceToHost, p->st));
    }
    BNM_CUDA_TRY(cudaStreamSynchronize(p->st));
    return BNM_OK;
}

extern "C" int bnm_mlp_loss_and_grads(bnm_mlp* p, const float* X, const float* T, int32_t n, float* loss,
                                      float* grads) {
    if (!p || !X || !T || n < 1 || n > p->max_batch) return bnm_fail_msg(BNM_EINVAL, "batch must be in [1, max_batch]");
    BNM_CUDA_TRY(cudaSetDevice(p->device));
    BNM_CUDA_TRY(cudaMemcpyAsync(p->xin, X, (size_t)n * p->in * 4, cudaMemcpyHostToDevice, p->st));
    BNM_CUDA_TRY(cudaMemcpyAsync(p->tgt, T, (size_t)n * p->out * 4, cudaMemcpyHostToDevice, p->st));
    int rc = forward(p, n);
    if (!rc) rc = backward(p, n);
    if (rc) return rc;
    if (loss) BNM_CUDA_TRY(cudaMemcpyAsync(loss, p->loss, 4, cudaMemcpyDeviceToHost, p->st));
    if (grads) BNM_CUDA_TRY(cudaMemcpyAsync(grads, p->g, (size_t)p->n_params * 4, cudaMemcpyDeviceToHost, p->st));
    BNM_CUDA_TRY(cudaStreamSynchronize(p->st));
    return BNM_OK;
}

extern "C" int bnm_mlp_train(bnm_mlp* p, const float* X, const float* Y, int32_t n, int32_t epochs, int32_t batch,
                             float lr, uint64_t shuffle_seed, float* loss_per_epoch) {
    if (!p || !X || !Y || n < 1 || batch < 1 || batch > p->max_batch || epochs < 0)
        return bnm_fail_msg(BNM_EINVAL, "bad training arguments");
    BNM_CUDA_TRY(cudaSetDevice(p->device));
    if (p->data_n < n) {
        if (p->data_x) {
            cudaFree(p->data_x);
            cudaFree(p->data_y);
        }
        BNM_CUDA_TRY(cudaMalloc(&p->data_x, (size_t)n * p->in * 4));
        BNM_CUDA_TRY(cudaMalloc(&p->data_y, (size_t)n * p->out * 4));
        p->data_n = n;
        p->allocs.push_back(p->data_x);
        p->allocs.push_back(p->data_y);
    }
    BNM_CUDA_TRY(cudaMemcpyAsync(p->data_x, X, (size_t)n * p->in * 4, cudaMemcpyHostToDevice, p->st));
    BNM_CUDA_TRY(cudaMemcpyAsync(p->data_y, Y, (size_t)n * p->out * 4, cudaMemcpyHostToDevice, p->st));
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::mt19937_64 gen(shuffle_seed);
    std::vector<float> losses;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int ep = 0; ep < epochs; ep++) {
        std::shuffle(order.begin(), order.end(), gen);
        double sum = 0.0;
        int nb = 0;
        for (int s = 0; s + batch <= n; s += batch) {  // full batches only
            BNM_CUDA_TRY(cudaMemcpyAsync(p->idx, order.data() + s, (size_t)batch * 4, cudaMemcpyHostToDevice, p->st));
            gather_rows_kernel<<<64, 256, 0, p->st>>>(p->data_x, p->idx, batch, p->in, p->xin);
            gather_rows_kernel<<<64, 256, 0, p->st>>>(p->data_y, p->idx, batch, p->out, p->tgt);
            int rc = forward(p, batch);
            if (!rc) rc = backward(p, batch);
            if (rc) return rc;
            p->adam_t++;
            const float c1 = 1.f - std::pow(b1, (float)p->adam_t), c2 = 1.f - std::pow(b2, (float)p->adam_t);
            adam_kernel<<<256, 256, 0, p->st>>>(p->w, p->g, p->m, p->v, p->w16, p->n_params, lr, b1, b2, eps, c1, c2);
            float l = 0.f;
            BNM_CUDA_TRY(cudaMemcpyAsync(&l, p->loss, 4, cudaMemcpyDeviceToHost, p->st));
            BNM_CUDA_TRY(cudaStreamSynchronize(p->st));  // the index buffer is reused next batch
            sum += l;
            nb++;
        }
        if (loss_per_epoch) loss_per_epoch[ep] = nb ? (float)(sum / nb) : 0.f;
    }
    BNM_CUDA_TRY(cudaGetLastError());
    return BNM_OK;
}

extern "C" int64_t bnm_mlp_num_params(const bnm_mlp* p) { return p ? p->n_params : 0; }

extern "C" int bnm_mlp_get_params(bnm_mlp* p, float* flat) {
    if (!p || !flat) return bnm_fail_msg(BNM_EINVAL, "null argument");
    BNM_CUDA_TRY(cudaSetDevice(p->device));
    BNM_CUDA_TRY(cudaMemcpy(flat, p->w, (size_t)p->n_params * 4, cudaMemcpyDeviceToHost));
    return BNM_OK;
}

extern "C" int bnm_mlp_set_params(bnm_mlp* p, const float* flat) {
    if (!p || !flat) return bnm_fail_msg(BNM_EINVAL, "null argument");
    BNM_CUDA_TRY(cudaSetDevice(p->device));
    BNM_CUDA_TRY(cudaMemcpy(p->w, flat, (size_t)p->n_params * 4, cudaMemcpyHostToDevice));
    // new parameters start a new optimisation: Adam's moments and step count restart
    BNM_CUDA_TRY(cudaMemsetAsync(p->m, 0, (size_t)p->n_params * 4, p->st));
    BNM_CUDA_TRY(cudaMemsetAsync(p->v, 0, (size_t)p->n_params * 4, p->st));
    p->adam_t = 0;
    to_bf16_kernel<<<256, 256, 0, p->st>>>(p->w, p->w16, p->n_params);
    BNM_CUDA_TRY(cudaStreamSynchronize(p->st));
    return BNM_OK;
}
